// launch.h -- host-side launchers of the fluid kernels (kernels.cu).  All launches go on the
// stream given; none synchronises.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "fluid_device.cuh"

namespace slf {

void launch_state_stats(const Params& p, const float4* pos, const float4* vel, Status* st, cudaStream_t s);
void launch_max_compression(const Params& p, const float* rho, Status* st, cudaStream_t s);

// counting sort by dense cell index; cells (cell-relative positions) optional
void launch_count_cells(const Params& p, const float4* pos, const int4* cells, int3 low, int3 span, uint32_t* count,
                        uint32_t* lin, uint32_t* slot, cudaStream_t s);
size_t scan_tiles(uint32_t m);
// exclusive scan of data[0, m) in place; data[m] receives the total.  tile_sums holds
// scan_tiles(m) + 1 entries.
void launch_exclusive_scan(uint32_t* data, uint32_t m, uint32_t* tile_sums, cudaStream_t s);
void launch_scatter_members(uint32_t n, const uint32_t* lin, const uint32_t* slot, const uint32_t* start,
                            const uint32_t* ids, uint32_t* members, cudaStream_t s);
void launch_rank_reorder(uint32_t n, const uint32_t* lin, const uint32_t* start, const uint32_t* members,
                         const uint32_t* ids_in, const float4* pos_in, const float4* vel_in, const float* rho_in,
                         const int4* cells_in, uint32_t* ids_out, float4* pos_out, float4* vel_out, float* rho_out,
                         int4* cells_out, const float2* warm_in, float2* warm_out, uint32_t skip_begin,
                         uint32_t skip_end, Status* st, uint32_t* dest,
                         cudaStream_t s);

// The list passes' walk order (PairLists::order) over the dense cell box `span` of a sort:
// start is the sort's cell table (volume + 1), bcount holds walk_order_keys(span) + 1 words,
// tile_sums scan_tiles(walk_order_keys(span)) + 1, order n.
size_t walk_order_keys(int3 span);
// Particle counts up to which the EXACT density pass and the WCSPH force pass, without terrain or
// coupled bodies, run a warp a particle (k_density_warp, k_wcsph_force_warp), which then needs no
// walk order: below one 256-thread block per SM (148 on B200) a thread a particle leaves SMs idle
// and each thread walks its candidates in one long chain of loads.  Measured: 8k particles at
// support 4, density 392 -> 92 us and force 218 -> 67 us; 250k and 1M particles at support 2,
// density 219 -> 547 us and 562 -> 2250 us, so larger scenes keep a thread a particle.
constexpr uint32_t kWarpPassMax = 32768u;
// Scenes at support 3 and more (hundreds of neighbours, thousands of candidates a particle) may
// keep the warp passes up to this many particles.  Off: on the 64k-particle scene at support 4
// the density pass gained (592 -> 548 us) but the force pass lost more (239 -> 358 us).
#ifndef SLF_WARP_PASS_WIDE_MAX
#define SLF_WARP_PASS_WIDE_MAX 0u
#endif
inline bool warp_rows(uint32_t n, float radius, float spacing) {
    return n <= kWarpPassMax || (n <= SLF_WARP_PASS_WIDE_MAX && radius >= 3.0f * spacing);
}
void launch_walk_order(uint32_t volume, int3 span, const uint32_t* start, uint32_t* bcount, uint32_t* tile_sums,
                       uint32_t* order, cudaStream_t s);

// pair passes: the density pass builds the substep's neighbour lists, the others walk them
// T: terrain regions (regions = 0: none); slope (optional): each particle's ground density gradient
void launch_density(const Params& p, const GridDev& fg, const GridDev& wg, const float4* pos, const float4* walls,
                    const PairLists& fl, const PairLists& wl, float* rho, float* press, float* scaled, float* alpha,
                    Status* st, const TerrainDev& T, float4* slope, cudaStream_t s, const MoverDev& M = MoverDev{});
// vel_pre (optional): the velocity before the wall clamp, its w lane the bits of the components
// the clamp zeroed (1 x, 2 y, 4 z), for the adjoint
void launch_wcsph_force(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                        const float4* pos, const float4* vel, const float* rho, const float* press,
                        const float* scaled, const float4* walls, float4* pos_out, float4* vel_out, Status* st,
                        float4* vel_pre, const TerrainDev& T, const float4* slope, cudaStream_t s,
                        const MoverDev& M = MoverDev{});
// coupled bodies: each particle's count of pairs whose damping a body takes (count[i]); then,
// with their exclusive scan in `offset` (n + 1 entries), the pairs' force and torque records and
// per (512-particle chunk, body) their sums in order (felt: chunks x bodies pairs of float4); and
// whether the last sort's table holds fluid in the cell box [lo, hi] (*wet set to 1, else left)
void launch_mover_count(const Params& p, const StepConsts* sc, const MoverDev& M, const float4* pos,
                        const float4* vel, const float* rho, const float* press, const float* scaled,
                        uint32_t* count, cudaStream_t s);
void launch_mover_felt(const Params& p, const StepConsts* sc, const MoverDev& M, const float4* pos, const float4* vel,
                       const float* rho, const float* press, const float* scaled, const float4* centre,
                       uint32_t bodies, const uint32_t* offset, float4* pair, float4* felt, cudaStream_t s);
// the bodies' felt records of a substep (launch_mover_felt) added into impulse[2 b] (force x dt)
// and impulse[2 b + 1] (torque x dt), chunk by chunk in order
void launch_mover_fold(uint32_t n, uint32_t bodies, const float4* felt, float dt, float4* impulse, cudaStream_t s);
void launch_cells_wet(const GridDev& g, int3 lo, int3 hi, uint32_t* wet, cudaStream_t s);
size_t rate_partial_bytes(uint32_t n);
// Looks up, once per process, how many blocks of the solver passes the device holds at once (not
// during a stream capture): their grids take no more, each block striding over rows.
void prepare_solver_grids();
// The same for the adjoint's stiffness passes (adjoint.cu) and the FAST check (kernels_fast.cu).
void prepare_adjoint_grids();
void prepare_fast_grids();
// One solver check: writes each particle's stiffness into the w lane of its position, and either
// sets st->settled or advances st->iterations.  Both it and the push do nothing once the solve
// has settled, so a batch of iterations can be queued ahead of the check that ends it.
// rec (optional): the check's rates and the velocities it read, recorded for the adjoint.
// loop (optional): the while-node handle of a solve captured as a CUDA graph; the check that
// stops the solve ends that loop, and the push bounds it at max_iterations + 1 bodies.
void launch_rate(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                 float4* pos, const float4* vel, const float* rho, const float* alpha, const float4* walls,
                 void* partials, Status* st, SolveRec rec, cudaStream_t s, unsigned long long loop = 0);
// applied (optional, stride 2): each particle's stiffness impulse sum, for warm starts
void launch_push(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, const float4* pos,
                 float4* vel, const float4* walls, Status* st, float* applied, cudaStream_t s,
                 unsigned long long loop = 0);
// warm start: pos.w = share * applied / dt, applied = that stiffness * dt
void launch_warm_kappa(const Params& p, const StepConsts* sc, float share, float* applied, float4* pos, cudaStream_t s);
void launch_viscous(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, const float4* pos,
                    const float4* vel, const float* rho, const float4* walls, float4* vel_out, cudaStream_t s);
void launch_advance(const Params& p, const StepConsts* sc, const float4* pos_in, float4* pos_out, float4* vel,
                    Status* st, float4* vel_pre, cudaStream_t s);

// neighbour lists on demand
void launch_list_count(const Params& p, const GridDev& g, const float4* pos, const float4* pts, uint32_t* counts,
                       cudaStream_t s);
void launch_list_fill(const Params& p, const GridDev& g, const float4* pos, const float4* pts, const uint32_t* start,
                      uint32_t* items, cudaStream_t s);

// domain
// keep flags: the domain's inside (drain = 0) or a drain box's outside (drain = 1)
// The k body points at `elapsed` sorted by (cell, owner, current place) into the *_out arrays,
// with the dense cell table of box (low, span) in table (volume + 1 entries, the last the total):
// lin, slot, members hold k entries, tiles scan_tiles(volume) + 1.  Every point's cell must lie
// in the box.
void launch_carry_movers(const Params& p, uint32_t k, const float4* start, const float4* vel, float elapsed, int3 low,
                         int3 span, uint32_t volume, uint32_t* lin, uint32_t* slot, uint32_t* table, uint32_t* tiles,
                         uint32_t* members, float4* start_out, float4* vel_out, float4* pos_out, cudaStream_t s);

// the particles inside any of `count` boxes (boxes: low, high pairs): keep flags, then (after an
// exclusive scan of them into `at`) their index, position and velocity in index order; and the
// velocities of listed particles written back
void launch_in_boxes(uint32_t n, const float4* pos, const float3* boxes, uint32_t count, uint32_t* keep, cudaStream_t s);
void launch_gather_kept(uint32_t n, const uint32_t* keep, const uint32_t* at, const float4* pos, const float4* vel,
                        uint32_t* index, float* pv, cudaStream_t s);
void launch_scatter_velocities(uint32_t m, const uint32_t* index, const float* v3, float4* vel, cudaStream_t s);
void launch_domain_flags(const Params& p, const float4* pos, const int4* cells, float3 low, float3 high, int drain,
                         uint32_t* keep, cudaStream_t s);
// emitters: mark the taken lattice slots (taken cleared, total + 1 words), then, after an
// exclusive scan of taken, write up to `room` particles for the free slots in slot order
void launch_emitter_taken(const Params& p, const float4* pos, const int4* cells, float3 low, int3 cnt, float spacing,
                          float clear, uint32_t* taken, cudaStream_t s);
void launch_emit(uint32_t total, const uint32_t* taken_ex, int3 cnt, float3 low, float spacing, float3 velocity,
                 uint32_t room, uint32_t first_id, float4* pos_out, float4* vel_out, uint32_t* ids_out, float* rho_out,
                 cudaStream_t s);
void launch_compact(uint32_t n, const uint32_t* keep, const uint32_t* dest, const uint32_t* ids_in,
                    const float4* pos_in, const float4* vel_in, const float* rho_in, const int4* cells_in,
                    uint32_t* ids_out, float4* pos_out, float4* vel_out, float* rho_out, int4* cells_out,
                    const float2* warm_in, float2* warm_out, cudaStream_t s);

void launch_set_consts(const StepConsts& c, StepConsts* out, cudaStream_t s);

// xyz triples <-> float4
void launch_pack3(uint32_t n, const float4* in, float* out, cudaStream_t s);
// bad (optional): incremented for each triple with a non finite component
void launch_unpack3(uint32_t n, const float* in, float4* out, cudaStream_t s, uint32_t* bad = nullptr);

// FAST arithmetic variants (kernels_fast.cu): same lists, order and sums, fused rounding; the
// lists hold indexes only (with the cell step in their top bits) and each pass recomputes the
// kernel gradient from the positions.  `cells` non-null (or `rel`) selects cell-relative
// positions: pos holds offsets in [0, r) from the cell corner, cells the integer cells.
void launch_density_fast(const Params& p, const GridDev& fg, const GridDev& wg, const float4* pos, const int4* cells,
                         const float4* walls, const PairLists& fl, const PairLists& wl, float* rho, float* press,
                         float* scaled, float* alpha, Status* st, cudaStream_t s);
void launch_wcsph_force_fast(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                             const float4* pos, const int4* cells, const float4* vel, const float* rho,
                             const float* press, const float* scaled, const float4* walls, float4* pos_out,
                             int4* cells_out, float4* vel_out, Status* st, float4* vel_pre, cudaStream_t s);
// the stiffness goes into pos.w, as in launch_rate
void launch_rate_fast(int which, bool rel, const Params& p, const StepConsts* sc, const PairLists& fl,
                      const PairLists& wl, float4* pos, const float4* vel, const float* rho, const float* alpha,
                      const float4* walls, void* partials, Status* st, SolveRec rec, cudaStream_t s,
                      unsigned long long loop = 0);
void launch_push_fast(bool rel, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                      const float4* pos, float4* vel, const float4* walls, Status* st, float* applied,
                      cudaStream_t s, unsigned long long loop = 0);
void launch_viscous_fast(bool rel, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                         const float4* pos, const float4* vel, const float* rho, const float4* walls,
                         float4* vel_out, cudaStream_t s);
void launch_advance_rel(const Params& p, const StepConsts* sc, const float4* pos_in, const int4* cells_in,
                        float4* pos_out, int4* cells_out, float4* vel, Status* st, float4* vel_pre, cudaStream_t s);
// absolute positions (xyz triples, or float4 when xyz is null) -> offsets and cells; and back.
// bad (optional): incremented for each position with a non finite component
void launch_to_relative(const Params& p, uint32_t n, const float* xyz, const float4* abs4, float4* pos, int4* cells,
                        cudaStream_t s, uint32_t* bad = nullptr);
void launch_from_relative(const Params& p, uint32_t n, const float4* pos, const int4* cells, float* xyz,
                          cudaStream_t s);
void launch_state_stats_rel(const Params& p, const int4* cells, const float4* vel, Status* st, cudaStream_t s);
// start null: counts into out[i]; else fills lists at start[i]
void launch_list_rel(const Params& p, const GridDev& g, const float4* pos, const int4* cells, const float4* pts,
                     const uint32_t* start, uint32_t* out, cudaStream_t s);

// `form` in the adjoint launchers: how the lists hold a neighbour, 1 EXACT {index, g} entries,
// 0 FAST index entries (absolute positions), 2 FAST entries with cell steps (cell-relative
// positions: pos then holds each particle's offset from its cell).
//
// The adjoint of one WCSPH substep (adjoint.cu).  Inputs are the recomputed forward of the
// substep (sorted positions and velocities, lists, densities, pressures, the pre-clamp velocity,
// the sort's destinations) and the adjoint of its output state xo, vo (sorted order); outputs
// the adjoint of its input state xp, vp in the order before the sort, and adds the parameter
// gradients (viscosity, wall viscosity, stiffness, gravity) to grads[kGradSlots].  T and slope:
// the terrain regions and the density pass's ground slopes (T.regions = 0: no terrain); bodies:
// the coupled bodies' points the substep met (count 0: none).
void launch_adjoint_wcsph(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                          int form, const float4* pos, const float4* vel, const float* rho, const float* press,
                          const float* scaled, const float4* walls, const float4* vel_pre, const uint32_t* dest,
                          const float4* xo, const float4* vo, float4* ab, float4* xb, float4* vb, float* rb,
                          float4* xp, float4* vp, double* grads, const TerrainDev& T, const float4* slope,
                          const MoverDev& bodies, cudaStream_t s);

// The adjoint of a DFSPH substep, in pieces the host strings together (adjoint.cu): the advance;
// one solver iteration (kappa, then the velocity adjoint before its push); the viscosity; the
// factors and the densities; and the way back through the sort.
void launch_adj_advance_dfsph(const Params& p, const StepConsts* sc, const float4* vel_pre, const float4* xo,
                              const float4* vo, float4* xb, float4* w, cudaStream_t s);
void launch_adj_iteration(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                          int form, const float4* pos, const float4* walls, const float4* w, const float* rate,
                          const float* alpha, const float* rho, const float4* vel, float4* kw, float4* vr,
                          float* abar, float* rb, float4* wout, float4* xb, cudaStream_t s, int parts = 3,
                          const float2* appbar = nullptr);
// warm starts: the adjoint of a solve's warm push (kappa_w = share applied / dt, applied the
// impulse of the particle's last solve of this kind, sorted): its kappa_w-bar from w, the push's
// position adjoint into xb, w through to wout, and applied-bar before the solve into component
// `which` of appbar_out (appbar: the adjoint of the impulse the solve leaves)
void launch_adj_warm(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                     int form, const float4* pos, const float4* walls, const float4* w, const float2* applied,
                     const float2* appbar, float share, float4* kw, float4* vr, float2* appbar_out, float4* wout,
                     float4* xb, cudaStream_t s);
void launch_adj_viscosity(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, int form,
                          const float4* pos, const float4* vel, const float* rho, const float* zeros,
                          const float4* walls, float4* w, float4* ab, float4* xb, float* rb, double* grads,
                          cudaStream_t s);
void launch_adj_factors_density(const Params& p, const PairLists& fl, const PairLists& wl, int form,
                                const float4* pos, const float4* walls, const float* alpha, const float* abar,
                                float4* gt, const float* rb, float4* xb, cudaStream_t s);
void launch_adj_unsort(uint32_t n, const uint32_t* dest, const float4* xb, const float4* vb, float4* xp, float4* vp,
                       cudaStream_t s, const float2* ib = nullptr, float2* ip = nullptr);

// kernels launched through this library by the process so far
uint64_t kernel_launches();
void note_launch();
// adds k (negative: takes back launches recorded into a graph, counted when it runs)
void note_launches(int64_t k);

// message slf_last_error() returns on this thread
void set_last_error(const std::string& message);

}  // namespace slf
