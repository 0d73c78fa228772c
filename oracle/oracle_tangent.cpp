// oracle_tangent.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The CPU restatement run in forward-mode FP64 derivative numbers (dual.hpp): one call builds a
// world with one box container (boundary.rs:41-68), adds the particles with the tangents of their
// positions and velocities, seeds the tangents of viscosity, sound speed and gravity, takes
// `steps` calls of step(dt) (step.rs:58-90) and returns the final state with its tangent.  Tests
// compare <g, tangent> with the CUDA library's adjoint through <g, J d> = <J^T g, d>.  Only tests/
// call it.

#include <cstdint>

#include "../include/solunar_fluid.h"
#include "fluid_oracle.hpp"

// f32::total_cmp's order on the value (the walls' sort key, boundary.rs:155-178)
inline bool total_less(Dual a, Dual b) { return oracle::total_less(a.v, b.v); }
inline uint64_t bits_of(Dual a) { return oracle::bits_of(a.v); }

using namespace oracle;

Settings settings_from_c(const slf_settings* s, int residual_sum);  // oracle_capi.cpp

extern "C" {

// pos, vel, dpos, dvel: n x 3 in the order the particles are added (ids 0..n-1); dparams: the
// tangents of viscosity, sound speed and gravity x, y, z.  Outputs in the world's final order,
// with out_ids naming each row.
int32_t orc_tangent_run(const slf_settings* s, int32_t residual_sum, const float* low, const float* high, uint64_t n,
                        const float* pos, const float* vel, const double* dpos, const double* dvel,
                        const double* dparams, uint32_t steps, float dt, double* out_pos, double* out_vel,
                        double* out_dpos, double* out_dvel, uint32_t* out_ids) {
    if (!s || !low || !high || !dparams || !out_pos || !out_vel || !out_dpos || !out_dvel || !out_ids)
        return INVALID_ARGUMENT;
    if (n && (!pos || !vel || !dpos || !dvel)) return INVALID_ARGUMENT;
    using V = V3<Dual>;
    World<Dual> w;
    Status st = World<Dual>::create(settings_from_c(s, residual_sum), w);
    if (st != OK) return st;
    for (int k = 0; k < 5; ++k) w.param_tangent[k] = dparams[k];
    st = w.add_box_container(V(Dual(low[0]), Dual(low[1]), Dual(low[2])),
                             V(Dual(high[0]), Dual(high[1]), Dual(high[2])), nullptr);
    if (st != OK) return st;
    for (uint64_t i = 0; i < n; ++i) {
        const float* p = pos + 3 * i;
        const float* v = vel + 3 * i;
        const double* dp = dpos + 3 * i;
        const double* dv = dvel + 3 * i;
        st = w.add_particle(V(Dual(p[0], dp[0]), Dual(p[1], dp[1]), Dual(p[2], dp[2])),
                            V(Dual(v[0], dv[0]), Dual(v[1], dv[1]), Dual(v[2], dv[2])), nullptr);
        if (st != OK) return st;
    }
    for (uint32_t k = 0; k < steps; ++k) {
        Report r;
        st = w.step(Dual(dt), r);
        if (st != OK) return st;
    }
    if (w.len() != n) return OUT_OF_RANGE;
    for (size_t i = 0; i < w.len(); ++i) {
        const V& p = w.positions[i];
        const V& v = w.velocities[i];
        double* op = out_pos + 3 * i;
        double* ov = out_vel + 3 * i;
        double* odp = out_dpos + 3 * i;
        double* odv = out_dvel + 3 * i;
        op[0] = p.x.v, op[1] = p.y.v, op[2] = p.z.v;
        odp[0] = p.x.d, odp[1] = p.y.d, odp[2] = p.z.d;
        ov[0] = v.x.v, ov[1] = v.y.v, ov[2] = v.z.v;
        odv[0] = v.x.d, odv[1] = v.y.d, odv[2] = v.z.d;
        out_ids[i] = w.ids[i];
    }
    return OK;
}

}  // extern "C"
