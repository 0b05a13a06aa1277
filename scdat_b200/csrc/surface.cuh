// surface.cuh -- the surface circuit of the body's faces: each face XMin..ZMax of the body box
// is a circuit node with capacitance C = eps0 eps_r A / d to the conducting core (the reference's
// capacitance per area, Toolkit/Surface Charging/src/DensePlasmaSurfaceCharging.cpp:6544-6552),
// an optional shunt conductance to ground and a linearised plasma current dI/dV.  Every step
// the charge the push collected on a face (exact fixed-point tallies) advances its potential by
// the implicit node update of SurfaceCircuitCoupling::advanceImplicit
// (Tools/Coupling/src/SurfaceCircuitCoupling.cpp:953-966):
//     (C/dt + G - dI/dV) V_new = C/dt V_old + I - dI/dV V_old,   I = dq/dt,
// which for G = dI/dV = 0 is the plain integration V += dq / C; the charge and potentials are
// kept in FP64.  The body's surface nodes then take the mean potential of the faces they lie on.
#pragma once

#include "common.cuh"

namespace scdat {

struct SurfaceDev {
    int32_t n;       // faces in the circuit (6)
    int32_t pad;
    double C[6];     // F
    double G[6];     // S to ground
    double didv[6];  // A/V
    double V[6];     // V
    double Q[6];     // C collected so far
    double I[6];     // A in the last step
};

// face k's update from the step's tallies (clears them)
__device__ __forceinline__ void surface_advance_face(SurfaceDev* S, LedgerDev* L, int k, double unit, double dt)
{
    const double dq = fx_to_double(L->patch_q[k][0], (long long)L->patch_q[k][1], unit);
    L->patch_q[k][0] = 0ull;
    L->patch_q[k][1] = 0ull;
    S->Q[k] += dq;
    const double I = dq / dt;
    S->I[k] = I;
    const double cdt = S->C[k] / dt, V = S->V[k];
    const double den = cdt + S->G[k] - S->didv[k];
    if (den > 0.0) S->V[k] = (cdt * V + I - S->didv[k] * V) / den;
}

// mean potential of the faces in `mask`, summed in ascending face order
__device__ __forceinline__ double surface_node_potential(const SurfaceDev* S, unsigned mask)
{
    double s = 0.0;
    int c = 0;
    for (int k = 0; k < 6; ++k)
        if ((mask >> k) & 1u) {
            s += S->V[k];
            ++c;
        }
    return c ? s / c : 0.0;
}

void launch_surface_advance(SurfaceDev* S, LedgerDev* L, double unit, double dt, cudaStream_t st);
void launch_surface_apply(const SurfaceDev* S, int64_t n, const int32_t* node, const uint8_t* mask, double* phi,
                          cudaStream_t st);

}  // namespace scdat
