// common.cuh -- device-side building blocks shared by the PIC-MCC kernels.
//
//  * 128-bit two's-complement fixed point accumulated with two 64-bit integer atomics, so
//    charge and ledger sums are exact and independent of thread order (deterministic).
//  * Philox4x32-10 counter-based RNG (Salmon et al., SC'11), keyed by (seed) with counter
//    (particle id, step, purpose): every particle owns its random stream.
//  * Flat views of the mesh, fields and particle store that the kernels take by value.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace scdat {

// ------------------------------------------------------------------------------------
// Fixed point: value = (hi * 2^64 + lo) * 2^-64 * unit, hi signed, lo unsigned.
// ------------------------------------------------------------------------------------
struct Fx128 {
    unsigned long long lo;
    long long hi;
};

__host__ __device__ inline Fx128 fx_from_double(double v)
{
    // v is already divided by the unit (a power of two, so the division is exact).
    double fl = floor(v);
    Fx128 r;
    r.hi = (long long)fl;
    double frac = v - fl;  // exact, in [0, 1)
#ifdef __CUDA_ARCH__
    r.lo = __double2ull_rz(frac * 18446744073709551616.0);
#else
    r.lo = (unsigned long long)(frac * 18446744073709551616.0);
#endif
    return r;
}

__host__ __device__ inline void fx_add(Fx128& a, const Fx128& b)
{
    unsigned long long lo = a.lo + b.lo;
    a.hi += b.hi + (lo < a.lo ? 1 : 0);
    a.lo = lo;
}

__host__ __device__ inline double fx_to_double(unsigned long long lo, long long hi, double unit)
{
    return (double)hi * unit + (double)lo * (unit * 5.421010862427522170037264e-20);  // 2^-64
}

__device__ inline void fx_atomic_add(unsigned long long* lo_acc, unsigned long long* hi_acc, const Fx128& v)
{
    if (v.lo == 0ull && v.hi == 0ll) return;
    unsigned long long old = atomicAdd(lo_acc, v.lo);
    unsigned long long carry = (old + v.lo < old) ? 1ull : 0ull;
    unsigned long long h = (unsigned long long)v.hi + carry;
    if (h) atomicAdd(hi_acc, h);
}

// A species' particle store as the re-sort gather sees it: six coordinate arrays (positions,
// then velocities), tet ids and particle ids.
template <typename T>
struct GatherArrays {
    T* v[6];
    int32_t* tet;
    uint32_t* id;
};


// Node charge accumulators of the FP64 form: each 128-bit contribution is split into 32-bit
// limbs that go into three 64-bit words with return-free atomic adds (no thread waits on an
// atomic), and the limbs are recombined exactly when the charge is read.  2^32 contributions
// per node and step fit before a limb could wrap.  The precision form uses l0 alone, as one
// word per node (fx_red_word), with l1 = h = nullptr.
struct ChargeAcc {
    unsigned long long* l0;  // bits 0..31 of each contribution
    unsigned long long* l1;  // bits 32..63
    unsigned long long* h;   // the signed high word
};

__device__ __forceinline__ void fx_red(const ChargeAcc& A, int node, const Fx128& v)
{
    unsigned long long a = v.lo & 0xffffffffull, b = v.lo >> 32;
    if (a) atomicAdd(A.l0 + node, a);
    if (b) atomicAdd(A.l1 + node, b);
    if (v.hi) atomicAdd(A.h + node, (unsigned long long)v.hi);
}

// The precision form's accumulators: one signed 64-bit word per node in units of 2^-36 of
// the charge unit.  Its contributions carry FP32 barycentric weights (24-bit mantissas), so
// this resolution loses nothing they hold, and each contribution is one return-free atomic
// (against three limb atomics).  A node's sum stays exact up to 2^27 unit charges per step.
constexpr double kWordScale = 68719476736.0;  // 2^36

__device__ __forceinline__ void fx_red_word(const ChargeAcc& A, int node, double v)
{
    const long long w = __double2ll_rn(v * kWordScale);
    if (w) atomicAdd(A.l0 + node, (unsigned long long)w);
}

// the word as a 128-bit value in units of 2^-64
__host__ __device__ inline Fx128 fx_from_word(unsigned long long w)
{
    const long long s = (long long)w;
    return Fx128{w << 28, s >> 36};
}

// A limb triple, or with l1 == nullptr a single word (the precision form's layout).
__host__ __device__ inline Fx128 fx_from_acc(const unsigned long long* l0, const unsigned long long* l1,
                                             const unsigned long long* h, int64_t i);

__host__ __device__ inline Fx128 fx_from_limbs(unsigned long long l0, unsigned long long l1, unsigned long long h)
{
    Fx128 r{l0, (long long)h};
    Fx128 m{l1 << 32, (long long)(l1 >> 32)};
    fx_add(r, m);
    return r;
}

__host__ __device__ inline Fx128 fx_from_acc(const unsigned long long* l0, const unsigned long long* l1,
                                             const unsigned long long* h, int64_t i)
{
    return l1 ? fx_from_limbs(l0[i], l1[i], h[i]) : fx_from_word(l0[i]);
}

// ------------------------------------------------------------------------------------
// Philox4x32-10
// ------------------------------------------------------------------------------------
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    }
}

// Two (0,1) doubles with 53-bit resolution for (seed; id, step, purpose).
__host__ __device__ inline void uniform2(uint64_t seed, uint64_t id, uint32_t step, uint32_t purpose, double& u0,
                                         double& u1)
{
    uint32_t c[4] = {(uint32_t)id, (uint32_t)(id >> 32), step, purpose};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t m0 = (((uint64_t)c[0] << 21) ^ (uint64_t)(c[1] >> 11)) & ((1ull << 53) - 1);
    uint64_t m1 = (((uint64_t)c[2] << 21) ^ (uint64_t)(c[3] >> 11)) & ((1ull << 53) - 1);
    u0 = ((double)m0 + 0.5) * (1.0 / 9007199254740992.0);
    u1 = ((double)m1 + 0.5) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------------------------------
// Device views
// ------------------------------------------------------------------------------------
constexpr double kBaryEps = 1e-8;        // PICParticleAlgorithms.cpp:286
constexpr double kMinTimeStep = 1e-20;   // PICParticleAlgorithms.cpp:583
constexpr int kMaxSubsteps = 100000;     // PICParticleAlgorithms.cpp:584
constexpr int kWalkSteps = 64;           // neighbour-walk cap before the grid lookup

// tet[] encoding of particle state: >= 0 active with that tet as location hint,
// -1 active without a hint, kTetAbsorbed / kTetEscaped inactive.
constexpr int32_t kTetNoHint = -1;
constexpr int32_t kTetAbsorbed = -2;
constexpr int32_t kTetEscaped = -3;

struct MeshView {
    int64_t N, T;
    const double* xyz;       // [N*3]
    const int4* tet;         // [T]
    const int4* nbr;         // [T] neighbour across the face opposite local vertex f
    const double* geom;      // [T*16] 128-byte records: J^-1 (row-major), origin xyz, 4 face
                             // neighbours and 4 node ids as int32
    const float* geomf;      // [T*12] the same in FP32 (mixed form), origin-relative
    const float* trec;       // [T*64] mixed-form 256-byte records (FP32 J^-1, nodal E, node ids,
                             // neighbours | FP32 origin offsets to the 4 neighbours)
    const double* erec;      // [T*12] FP64 nodal E of each tet's 4 nodes (refreshed per solve)
    // locate grid: uniform bins over the bounding box, tets listed by ascending id
    double gmin[3];
    double ginv[3];
    int32_t gdim[3];
    double gdelta;           // query half-width covering the containment tolerance
    const int32_t* bin_start;
    const int32_t* bin_tets;
    double bmin[3], bmax[3];  // domain bounds (PICCycle.cpp:1039-1066)
    int32_t use_nbr;
};

struct LedgerDev {
    // 7 rows x {qe_lo, qe_hi, qi_lo, qi_hi, en_lo, en_hi, n_e, n_i}
    unsigned long long row[7][8];
    unsigned long long surf_lo, surf_hi;     // surface_deposited_charge
    unsigned long long substeps, lost_events, mcc_hits, active;
    unsigned long long flags;                // device error flag word
    unsigned long long lsq_bad;              // bit 8: the nodal field had a non-finite value
    unsigned long long pad[4];
    // charge [fixed point lo, hi] and count of particles lost into each face XMin..ZMax of the
    // body box this step (surface circuit; cleared when the circuit advances)
    unsigned long long patch_q[6][2];
    unsigned long long patch_n[6];
    // charge of the secondary electrons emitted per ledger row (fixed point lo, hi)
    unsigned long long emit_q[7][2];
};

enum DeviceFlag : unsigned long long {
    kFlagBadTet = 1ull << 0,
    kFlagPcgNotConverged = 1ull << 1,
    kFlagDeferOverflow = 1ull << 2,  // a stay-first pass 1 found its deferred list full
};

struct SpeciesDev {
    double q, m, w, qm;
    double cw_seg;       // (q / nseg) * w, the reference's per-point charge weight
    int32_t electron_like;
    int32_t mcc_enabled;
    int32_t mcc_mode;
    int32_t pad;
    double mcc_n, mcc_sigma, mcc_eref, mcc_alpha, mcc_eth;
    // null-collision MCC (mode 2): the species' largest speed at the end of the previous push
    // ([0], float bits; 0 = none yet) and of the current one ([1], raised by the push)
    unsigned* vmax;
};

// splitmix64's output mix (Steele, Lea and Flood, OOPSLA 2014), a bijection of 64-bit words.
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}

// A (0,1) double with 53-bit resolution for (seed; id, step): the null-collision selection
// draw, a counter-based stream distinct from the Philox streams (one multiply-mix chain
// instead of ten Philox rounds, since every particle draws it every step).
__host__ __device__ inline double select_uniform(uint64_t seed, uint32_t id, uint32_t step)
{
    const uint64_t key = ((uint64_t)step << 32) | (uint64_t)id;
    const uint64_t z = mix64(mix64(seed ^ 0x5CDA7B2005CDA7B2ull) + key * 0x9E3779B97F4A7C15ull);
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

struct PushParams {
    double dt;
    double floor_ratio;
    int32_t nseg;
    int32_t dep_kernel;
    int32_t face_bc[6];
    double period[3];
    int32_t body_tally;
    int32_t do_mcc;
    double otol, ntol;
    double inv_uq, inv_ue;   // 1 / fixed-point units for charge and energy
    uint64_t seed;
    uint32_t step;
    int32_t deposit;
    // surface circuit: particles lost into the body box [blo, bhi] are tallied per face
    int32_t patches;
    int32_t see_model;       // secondary emission of electrons collected by the body: 0 off,
                             // 1 Sternglass, 2 Whipple, 3 Sims, 4 Katz (the legacy yields)
    double blo[3], bhi[3];
    double see_dmax, see_emax_ev;
    double see_sims_n, see_sims_xm;  // Sims: exponent (>= 1.05) and the root xm it implies
    double see_katz[4];              // Katz: range coefficients r1, n1, r2, n2
};

}  // namespace scdat
