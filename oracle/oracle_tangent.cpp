// oracle_tangent.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The CPU restatement run in forward-mode derivative numbers (dual.hpp): one call builds a world
// with one box container (boundary.rs:41-68), adds the particles with the tangents of their
// positions and velocities, seeds the tangents of viscosity, sound speed and gravity, takes
// `steps` calls of step(dt) (step.rs:58-90) and returns the final state with its tangent.  With
// precision 32 the values are the float restatement's bit for bit (the FP32 program the CUDA
// library runs); with 64 they are the FP64 method's.  Tests compare <g, tangent> with the CUDA
// library's adjoint through <g, J d> = <J^T g, d>.  Only tests/ call it.

#include <cstdint>

#include "../include/solunar_fluid.h"
#include "fluid_oracle.hpp"

// f32::total_cmp's order and the bit pattern of the value (the walls' sort key, boundary.rs:155-178)
template <class V, class D> inline bool total_less(DualOf<V, D> a, DualOf<V, D> b) {
    return oracle::total_less(a.v, b.v);
}
template <class V, class D> inline uint64_t bits_of(DualOf<V, D> a) { return oracle::bits_of(a.v); }

using namespace oracle;

Settings settings_from_c(const slf_settings* s, int residual_sum);  // oracle_capi.cpp

namespace {

uint32_t g_hold = 0;  // World::hold of the next runs (orc_tangent_hold)

template <class V, class D = double>
int32_t tangent_run(const slf_settings* s, int32_t residual_sum, const float* low, const float* high, uint64_t n,
                    const float* pos, const float* vel, const double* dpos, const double* dvel, const double* dparams,
                    uint32_t steps, float dt, const uint32_t* forced, uint64_t nforced, double* out_pos,
                    double* out_vel, double* out_dpos, double* out_dvel, uint32_t* out_ids) {
    using R = DualOf<V, D>;
    using Vec = V3<R>;
    World<R> w;
    Status st = World<R>::create(settings_from_c(s, residual_sum), w);
    if (st != OK) return st;
    for (int k = 0; k < 5; ++k) w.param_tangent[k] = dparams[k];
    w.forced_iterations.assign(forced, forced + nforced);
    w.hold = g_hold;
    st = w.add_box_container(Vec(R(low[0]), R(low[1]), R(low[2])), Vec(R(high[0]), R(high[1]), R(high[2])), nullptr);
    if (st != OK) return st;
    for (uint64_t i = 0; i < n; ++i) {
        const float* p = pos + 3 * i;
        const float* v = vel + 3 * i;
        const double* dp = dpos + 3 * i;
        const double* dv = dvel + 3 * i;
        st = w.add_particle(Vec(R(p[0], dp[0]), R(p[1], dp[1]), R(p[2], dp[2])),
                            Vec(R(v[0], dv[0]), R(v[1], dv[1]), R(v[2], dv[2])), nullptr);
        if (st != OK) return st;
    }
    for (uint32_t k = 0; k < steps; ++k) {
        Report r;
        st = w.step(R(dt), r);
        if (st != OK) return st;
    }
    if (w.len() != n) return OUT_OF_RANGE;
    for (size_t i = 0; i < w.len(); ++i) {
        const Vec& p = w.positions[i];
        const Vec& v = w.velocities[i];
        double* op = out_pos + 3 * i;
        double* ov = out_vel + 3 * i;
        double* odp = out_dpos + 3 * i;
        double* odv = out_dvel + 3 * i;
        op[0] = double(p.x.v), op[1] = double(p.y.v), op[2] = double(p.z.v);
        odp[0] = double(p.x.d), odp[1] = double(p.y.d), odp[2] = double(p.z.d);
        ov[0] = double(v.x.v), ov[1] = double(v.y.v), ov[2] = double(v.z.v);
        odv[0] = double(v.x.d), odv[1] = double(v.y.d), odv[2] = double(v.z.d);
        out_ids[i] = w.ids[i];
    }
    return OK;
}

}  // namespace

extern "C" {

// The quantities the next tangent runs hold constant (World::hold bits; 0: none).
void orc_tangent_hold(uint32_t mask) { g_hold = mask; }

// precision: 32 (values of the float restatement, bit for bit), 64 (the FP64 method) or -32 (the
// float restatement's values with every derivative operation rounded to float).
// pos, vel, dpos, dvel: n x 3 in the order the particles are added (ids 0..n-1); dparams: the
// tangents of viscosity, sound speed and gravity x, y, z.  forced (nforced counts, may be 0): the
// iteration counts the DFSPH solves take, divergence and density of each substep in turn, so that
// the run differentiates the discrete steps another run took.  Outputs in the world's final
// order, with out_ids naming each row.
int32_t orc_tangent_run(const slf_settings* s, int32_t precision, int32_t residual_sum, const float* low,
                        const float* high, uint64_t n, const float* pos, const float* vel, const double* dpos,
                        const double* dvel, const double* dparams, uint32_t steps, float dt, const uint32_t* forced,
                        uint64_t nforced, double* out_pos, double* out_vel, double* out_dpos, double* out_dvel,
                        uint32_t* out_ids) {
    if (!s || !low || !high || !dparams || !out_pos || !out_vel || !out_dpos || !out_dvel || !out_ids)
        return INVALID_ARGUMENT;
    if ((n && (!pos || !vel || !dpos || !dvel)) || (nforced && !forced)) return INVALID_ARGUMENT;
    if (precision == 32)
        return tangent_run<float>(s, residual_sum, low, high, n, pos, vel, dpos, dvel, dparams, steps, dt, forced,
                                  nforced, out_pos, out_vel, out_dpos, out_dvel, out_ids);
    if (precision == -32)
        return tangent_run<float, float>(s, residual_sum, low, high, n, pos, vel, dpos, dvel, dparams, steps, dt,
                                         forced, nforced, out_pos, out_vel, out_dpos, out_dvel, out_ids);
    if (precision == 64)
        return tangent_run<double>(s, residual_sum, low, high, n, pos, vel, dpos, dvel, dparams, steps, dt, forced,
                                   nforced, out_pos, out_vel, out_dpos, out_dvel, out_ids);
    return INVALID_ARGUMENT;
}

}  // extern "C"
