// Finite-volume building blocks of the ion fluids (device functions shared by the
// reference-signature entry points and the fused step).
#pragma once
#include <climits>

#include "common.cuh"

namespace mhd
{
constexpr int kMaxSpecies = 16;

// Per-launch parameters of the fluid kernels (all species of one launch share the mesh).
struct FluidParams
{
    int nsp;                        // species in this launch
    int limit;                      // Barth-Jespersen on/off
    double gamma, rel_limit, rho_floor, p_floor;
    Prim5 fs[kMaxSpecies];          // free-stream (inflow ghost) state per species
    int8_t absorb[kMaxSpecies];     // wall ghost: 1 = absorbing floor state, 0 = slip reflection
    // the caller's Dirichlet wall states (null: none): per face the slot of its state, -1 where the face
    // keeps ghost_state; wall_prim[(s * wall_n + slot) * 5 + m] the primitives of species s (this launch's)
    const int32_t *wall_slot = nullptr;
    const double *wall_prim = nullptr;
    int64_t wall_n = 0;
    // switch log (null: off).  Per entity a running hash of the discrete choices that the kernels make, so
    // that two runs can be compared entity by entity: the limiter's active bound per variable
    // [(s * 5 + q) * nc + c], the Rusanov wave speed and face-state fallbacks per face [s * nf + f] (species
    // of this launch), the floors of the update per cell [s * nc + c] (all species)
    uint32_t *sw_lim = nullptr, *sw_flux = nullptr, *sw_floor = nullptr;
};

// one step of the switch log's running hash (FNV-1a over 32-bit words)
__device__ __forceinline__ uint32_t sw_step(uint32_t h, uint32_t v) { return (h ^ v) * 16777619u; }
__device__ __forceinline__ void sw_log(uint32_t *log, int64_t i, uint32_t v) { log[i] = sw_step(log[i], v); }

// The limiter's choice for one variable (Barth-Jespersen psi = clamp(min(1, (hi - w)/dpos, (lo - w)/dneg,
// rel w / max(dpos, -dneg)), 0, 1)): which term sets psi (0: none, psi >= 1; 1: the upper bound; 2: the lower
// bound; 3: the relative limit; 4: psi <= 0) with the neighbour slot that gives the bound and the face slot of
// the extreme dl (7: the cell itself), the quantities that the limited gradient's derivative follows.  The
// quotients are formed as the kernels form them, so the comparison with psi is exact.
__device__ __forceinline__ uint32_t limiter_code(double psi, double wc, double lo, double hi, double dpos, double dneg, int jlo,
                                                 int jhi, int jpos, int jneg, double rel, bool rel_on)
{
    if (!(psi > 0.0)) return 4u;
    if (psi >= 1.0) return 0u;
    if (dpos > 1e-300 && psi == (hi - wc) / dpos) return 1u | uint32_t(jhi & 15) << 3 | uint32_t(jpos & 15) << 7;
    if (dneg < -1e-300 && psi == (lo - wc) / dneg) return 2u | uint32_t(jlo & 15) << 3 | uint32_t(jneg & 15) << 7;
    if (rel_on) return 3u | uint32_t((dpos >= -dneg ? jpos : jneg) & 15) << 3 | (dpos >= -dneg ? 0u : 1u) << 7;
    return 5u;
}

// Species-indexed strided field: value(s, i, m) = p[s * ss + i * si + m * sm]
template <class T> struct SField
{
    T *p;
    int64_t ss, si, sm;
    __device__ __forceinline__ T &operator()(int s, int64_t i, int m) const { return p[s * ss + i * si + m * sm]; }
};

// mhd::to_prim (Common/physics/Euler.h:13-21)
__device__ __forceinline__ Prim5 to_prim(double U0, double U1, double U2, double U3, double U4, double gamma, double rho_floor,
                                         double p_floor)
{
    Prim5 W;
    W.rho = dmax(U0, rho_floor);
    W.u = U1 / W.rho;
    W.v = U2 / W.rho;
    W.w = U3 / W.rho;
    const double ke = 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    W.p = dmax((gamma - 1.0) * (U4 - ke), p_floor);
    return W;
}

// mhd::ghost_state (Common/fluid/Reconstruction.cpp:9-24): kind 1 wall, 2 inflow, else zero gradient
__device__ __forceinline__ Prim5 ghost_state(int kind, bool absorb, const Prim5 &in, V3 n, const Prim5 &fs)
{
    if (kind == 1)
    {
        if (absorb) return Prim5{1e-12, 0, 0, 0, 1e-12};
        const double un = in.u * n.x + in.v * n.y + in.w * n.z;
        Prim5 g = in;
        g.u -= 2 * un * n.x;
        g.v -= 2 * un * n.y;
        g.w -= 2 * un * n.z;
        return g;
    }
    if (kind == 2) return fs;
    return in;
}

__device__ __forceinline__ void prim_arr(const Prim5 &w, double *a)
{
    a[0] = w.rho; a[1] = w.u; a[2] = w.v; a[3] = w.w; a[4] = w.p;
}

// The Dirichlet wall ghost of a GhostFn (Common/fluid/Reconstruction.h:21) as the ten-ion solver builds it
// (MarsUns/driver/MarsSolver.cpp:124-128 over its cached wall_state_, :147-165): on a listed wall face the
// ghost of species s is the caller's state whatever the inside state.  Null where the face keeps ghost_state.
__device__ __forceinline__ const double *wall_ghost(const FluidParams &p, int kind, int32_t f, int s)
{
    if (kind != 1 || !p.wall_slot) return nullptr;
    const int32_t k = p.wall_slot[f];
    return k < 0 ? nullptr : p.wall_prim + 5 * ((int64_t)s * p.wall_n + k);
}

// mhd::rusanov (Common/physics/Euler.h:30-49): flux per unit area through unit normal n (L -> R)
__device__ __forceinline__ void rusanov(const Prim5 &L, const Prim5 &R, V3 n, double gamma, double *F)
{
    auto cons = [&](const Prim5 &W, double *U) {
        U[0] = W.rho; U[1] = W.rho * W.u; U[2] = W.rho * W.v; U[3] = W.rho * W.w;
        U[4] = W.p / (gamma - 1.0) + 0.5 * W.rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    };
    double UL[5], UR[5];
    cons(L, UL);
    cons(R, UR);
    const double unL = L.u * n.x + L.v * n.y + L.w * n.z, unR = R.u * n.x + R.v * n.y + R.w * n.z;
    const double FL[5] = {L.rho * unL, L.rho * unL * L.u + L.p * n.x, L.rho * unL * L.v + L.p * n.y, L.rho * unL * L.w + L.p * n.z,
                          unL * (UL[4] + L.p)};
    const double FR[5] = {R.rho * unR, R.rho * unR * R.u + R.p * n.x, R.rho * unR * R.v + R.p * n.y, R.rho * unR * R.w + R.p * n.z,
                          unR * (UR[4] + R.p)};
    const double sL = fabs(unL) + sqrt(gamma * L.p / L.rho);
    const double sR = fabs(unR) + sqrt(gamma * R.p / R.rho);
    const double s = dmax(sL, sR);
    for (int q = 0; q < 5; ++q) F[q] = 0.5 * (FL[q] + FR[q]) - 0.5 * s * (UR[q] - UL[q]);
}

// Rusanov's choices: which side's wave speed is the larger (bit 0: R), the sign of that side's normal velocity
// (bit 1: negative), the wave speeds formed as rusanov forms them.  None where the two states are one state
// (a zero-gradient ghost): there the wave speed multiplies U_R - U_L = 0 and no choice reaches the flux.
// mirror (a slip wall's reflected ghost): the two speeds are one speed up to the rounding of the reflection,
// so only the sign of the normal velocity is a choice there.
__device__ __forceinline__ uint32_t rusanov_code(const Prim5 &L, const Prim5 &R, V3 n, double gamma, bool mirror)
{
    if (L.rho == R.rho && L.u == R.u && L.v == R.v && L.w == R.w && L.p == R.p) return 0u;
    const double unL = L.u * n.x + L.v * n.y + L.w * n.z, unR = R.u * n.x + R.v * n.y + R.w * n.z;
    if (mirror) return unL < 0.0 ? 2u : 0u;
    const double sL = fabs(unL) + sqrt(gamma * L.p / L.rho);
    const double sR = fabs(unR) + sqrt(gamma * R.p / R.rho);
    const bool r = sL < sR;
    return (r ? 1u : 0u) | ((r ? unR : unL) < 0.0 ? 2u : 0u);
}

// face_state of Common/fluid/FluxRHS.cpp:16-27: linear extrapolation with positivity fallback
__device__ __forceinline__ Prim5 face_state(const Prim5 &w, const double *g, V3 dx)
{
    Prim5 r;
    r.rho = w.rho + g[0] * dx.x + g[1] * dx.y + g[2] * dx.z;
    r.u = w.u + g[3] * dx.x + g[4] * dx.y + g[5] * dx.z;
    r.v = w.v + g[6] * dx.x + g[7] * dx.y + g[8] * dx.z;
    r.w = w.w + g[9] * dx.x + g[10] * dx.y + g[11] * dx.z;
    r.p = w.p + g[12] * dx.x + g[13] * dx.y + g[14] * dx.z;
    return (r.rho > 0 && r.p > 0) ? r : w;
}

// whether face_state falls back to the cell value (the same extrapolation of rho and p)
__device__ __forceinline__ bool face_state_fallback(const Prim5 &w, const double *g, V3 dx)
{
    const double rho = w.rho + g[0] * dx.x + g[1] * dx.y + g[2] * dx.z;
    const double p = w.p + g[12] * dx.x + g[13] * dx.y + g[14] * dx.z;
    return !(rho > 0 && p > 0);
}
// Slot map of the caller's wall states: slot[f] = i for faces[i] (device ids), -1 elsewhere (slot holds nf
// entries).  Throws unless every listed face is a distinct face of kind wall.
void build_wall_slots(const MeshView &m, const int32_t *faces, int32_t n, int32_t *slot, cudaStream_t s);
} // namespace mhd
