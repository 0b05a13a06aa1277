// field_kern.cuh -- bodies of the field-solve kernels (field.cu wraps each in a __global__
// of the same name without "_body"; the batched step runs them per scenario).  Every body takes
// the block's index and the block count of its grid-stride loop as a Grid, so one launch can
// give each scenario its own share of the blocks.
#pragma once

#include "field.cuh"

namespace scdat {

struct Grid {
    unsigned b, n;  // this block's index and the number of blocks working on the same arrays
};


// ---------------------------------------------------------------------------------------
// Deterministic block reduction helpers
// ---------------------------------------------------------------------------------------
template <int NV>
__device__ inline void block_sum(double (&v)[NV], double* sh /* [NV*32] */)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sh[k * 32 + w];
            v[k] = s;
        }
    }
}

// Writes this block's partials, and returns true in thread 0 of the last block to finish,
// with v[k] the sum over all blocks.  The last block sums the partials with all its threads
// (thread t takes blocks t, t+256, ...) and a fixed-shape tree, so the order is the same on
// every run.  Blocks have 256 threads.
template <int NV>
__device__ inline bool last_block(double (&v)[NV], double* part, unsigned int* ticket, Grid g)
{
    __shared__ bool am_last;
    __shared__ double red[NV][256];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) part[k * g.n + g.b] = v[k];
        __threadfence();
        unsigned int t = atomicInc(ticket, g.n - 1);
        am_last = (t == g.n - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = 0.0;
        for (unsigned int b = threadIdx.x; b < g.n; b += blockDim.x) s += __ldcg(part + k * g.n + b);
        red[k][threadIdx.x] = s;
    }
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
#pragma unroll
            for (int k = 0; k < NV; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = red[k][0];
    return true;
}

// ---------------------------------------------------------------------------------------
// Charge finalisation
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void k_finalize_rho_body(int64_t N, int S, const unsigned long long* __restrict__ l0,
                               const unsigned long long* __restrict__ l1, const unsigned long long* __restrict__ h,
                               double unit, double* __restrict__ rho, unsigned long long* total_lo,
                               unsigned long long* total_hi, Grid g)
{
    Fx128 tot{0ull, 0ll};
    for (int64_t n = g.b * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)g.n * blockDim.x) {
        Fx128 a{0ull, 0ll};
        for (int s = 0; s < S; ++s) fx_add(a, fx_from_acc(l0, l1, h, s * N + n));
        rho[n] = fx_to_double(a.lo, a.hi, unit);
        fx_add(tot, a);
    }
    // exact 128-bit reduction: warp shuffles of (lo, hi) pairs keep exactness
    for (int o = 16; o > 0; o >>= 1) {
        Fx128 b;
        b.lo = __shfl_down_sync(0xffffffffu, tot.lo, o);
        b.hi = __shfl_down_sync(0xffffffffu, tot.hi, o);
        fx_add(tot, b);
    }
    if ((threadIdx.x & 31) == 0) fx_atomic_add(total_lo, total_hi, tot);
}

__device__ __forceinline__ void k_species_rho_body(int64_t N, const unsigned long long* __restrict__ l0,
                              const unsigned long long* __restrict__ l1, const unsigned long long* __restrict__ h,
                              double unit, double* __restrict__ out, Grid g)
{
    for (int64_t n = g.b * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)g.n * blockDim.x) {
        Fx128 a = fx_from_acc(l0, l1, h, n);
        out[n] = fx_to_double(a.lo, a.hi, unit);
    }
}

// ---------------------------------------------------------------------------------------
// Right-hand side on the reduced rows
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void k_rhs_body(PoissonView A, const double* __restrict__ rho, const double* __restrict__ phi, double sign,
                      double* __restrict__ b, Grid g)
{
    for (int r = g.b * blockDim.x + threadIdx.x; r < A.R; r += g.n * blockDim.x) {
        int n = A.row_node[r];
        double bi = sign * rho[n] * A.cv[r];
        for (int e = A.lift_ptr[r]; e < A.lift_ptr[r + 1]; ++e) bi -= A.lift_val[e] * phi[A.lift_node[e]];
        b[r] = bi;
    }
}

// x (row space) <- phi, and phi <- x after the solve
__device__ __forceinline__ void k_gather_rows_body(PoissonView A, const double* __restrict__ phi, double* __restrict__ x, Grid g)
{
    for (int r = g.b * blockDim.x + threadIdx.x; r < A.R; r += g.n * blockDim.x) x[r] = phi[A.row_node[r]];
}

__device__ __forceinline__ void k_scatter_rows_body(PoissonView A, const double* __restrict__ x, double* __restrict__ phi, Grid g)
{
    for (int r = g.b * blockDim.x + threadIdx.x; r < A.R; r += g.n * blockDim.x) phi[A.row_node[r]] = x[r];
}

// ---------------------------------------------------------------------------------------
// PCG (FP64 values, or FP32 values for the inner solve of the mixed form)
// ---------------------------------------------------------------------------------------
// diagonal and its reciprocal in the precision of the solve
template <typename V> __device__ __forceinline__ double diag_at(const PoissonView& A, int i);
template <> __device__ __forceinline__ double diag_at<double>(const PoissonView& A, int i) { return A.diag[i]; }
template <> __device__ __forceinline__ double diag_at<float>(const PoissonView& A, int i) { return (double)A.diagf[i]; }
template <typename V> __device__ __forceinline__ double dinv_at(const PoissonView& A, int i);
template <> __device__ __forceinline__ double dinv_at<double>(const PoissonView& A, int i) { return A.dinv[i]; }
template <> __device__ __forceinline__ double dinv_at<float>(const PoissonView& A, int i) { return (double)A.dinvf[i]; }

template <typename V>
__device__ __forceinline__ double spmv_row(const PoissonView& A, const V* __restrict__ val, int r,
                                           const V* __restrict__ xv)
{
    double s = diag_at<V>(A, r) * (double)xv[r];
    for (int e = A.row_ptr[r]; e < A.row_ptr[r + 1]; ++e) s += (double)val[e] * (double)xv[A.col[e]];
    return s;
}

// r = b - A x, z = r / d, and the dots rz, rr, bb
template <typename V>
__device__ __forceinline__ void k_pcg_init_body(PoissonView A, const V* __restrict__ val, const V* __restrict__ b, const V* __restrict__ x,
                           V* __restrict__ r, V* __restrict__ z, PcgScalars* sc, double* part, Grid g)
{
    double acc[3] = {0.0, 0.0, 0.0};
    for (int i = g.b * blockDim.x + threadIdx.x; i < A.R; i += g.n * blockDim.x) {
        double ri = (double)b[i] - spmv_row(A, val, i, x);
        double zi = ri * dinv_at<V>(A, i);
        r[i] = (V)ri;
        z[i] = (V)zi;
        acc[0] += ri * zi;
        acc[1] += ri * ri;
        acc[2] += (double)b[i] * (double)b[i];
    }
    __shared__ double sh[3 * 32];
    block_sum<3>(acc, sh);
    if (last_block<3>(acc, part, &sc->ticket, g)) {
        sc->rz = acc[0];
        sc->rr = acc[1];
        sc->bb = acc[2];
        sc->rz_prev = 1.0;
        sc->iter = 0;
        double thr = sc->rtol * sc->rtol * (acc[2] > 0.0 ? acc[2] : 1.0);
        if (sc->abs_thr2 > 0.0) thr = sc->abs_thr2;
        sc->thr2 = thr;
        sc->done = (acc[1] <= thr || sc->max_iter <= 0) ? 1 : 0;
    }
}

// pn = z + beta p ; q = A pn ; dot pn.q
template <typename V>
__device__ __forceinline__ void k_pcg_spmv_body(PoissonView A, const V* __restrict__ val, const V* __restrict__ z, const V* __restrict__ p,
                           V* __restrict__ pn, V* __restrict__ q, PcgScalars* sc, double* part, Grid g)
{
    if (sc->done) return;
    const bool first = sc->iter == 0;
    const double beta = first ? 0.0 : sc->rz / sc->rz_prev;
    double acc[1] = {0.0};
    for (int i = g.b * blockDim.x + threadIdx.x; i < A.R; i += g.n * blockDim.x) {
        double pi = first ? (double)z[i] : (double)z[i] + beta * (double)p[i];
        double s = diag_at<V>(A, i) * pi;
        for (int e = A.row_ptr[i]; e < A.row_ptr[i + 1]; ++e) {
            int c = A.col[e];
            double pc = first ? (double)z[c] : (double)z[c] + beta * (double)p[c];
            s += (double)val[e] * pc;
        }
        pn[i] = (V)pi;
        q[i] = (V)s;
        acc[0] += pi * s;
    }
    __shared__ double sh[32];
    block_sum<1>(acc, sh);
    if (last_block<1>(acc, part, &sc->ticket, g)) sc->pq = acc[0];
}

// x += alpha pn ; r -= alpha q ; z = r / d ; dots rz, rr ; convergence test
template <typename V>
__device__ __forceinline__ void k_pcg_update_body(PoissonView A, V* __restrict__ x, const V* __restrict__ pn, V* __restrict__ r,
                             const V* __restrict__ q, V* __restrict__ z, PcgScalars* sc, double* part, Grid g)
{
    if (sc->done) return;
    const double pq = sc->pq;
    const double alpha = pq > 0.0 ? sc->rz / pq : 0.0;
    double acc[2] = {0.0, 0.0};
    for (int i = g.b * blockDim.x + threadIdx.x; i < A.R; i += g.n * blockDim.x) {
        double xi = (double)x[i] + alpha * (double)pn[i];
        double ri = (double)r[i] - alpha * (double)q[i];
        double zi = ri * dinv_at<V>(A, i);
        x[i] = (V)xi;
        r[i] = (V)ri;
        z[i] = (V)zi;
        acc[0] += ri * zi;
        acc[1] += ri * ri;
    }
    __shared__ double sh[2 * 32];
    block_sum<2>(acc, sh);
    if (last_block<2>(acc, part, &sc->ticket, g)) {
        sc->rz_prev = sc->rz;
        sc->rz = acc[0];
        sc->rr = acc[1];
        sc->iter += 1;
        if (acc[1] <= sc->thr2 || sc->iter >= sc->max_iter || !(pq > 0.0)) sc->done = 1;
    }
}

// FP64 residual of the refinement loop: r64 = b - A64 x64, and the dots rr, bb
__device__ __forceinline__ void k_residual64_body(PoissonView A, const double* __restrict__ b, const double* __restrict__ x,
                             double* __restrict__ r, float* __restrict__ rf, PcgScalars* sc, double* part, Grid g)
{
    double acc[2] = {0.0, 0.0};
    for (int i = g.b * blockDim.x + threadIdx.x; i < A.R; i += g.n * blockDim.x) {
        double ri = b[i] - spmv_row(A, A.val, i, x);
        r[i] = ri;
        rf[i] = (float)ri;
        acc[0] += ri * ri;
        acc[1] += b[i] * b[i];
    }
    __shared__ double sh[2 * 32];
    block_sum<2>(acc, sh);
    if (last_block<2>(acc, part, &sc->ticket, g)) {
        sc->rr = acc[0];
        sc->bb = acc[1];
    }
}

__device__ __forceinline__ void k_add_correction_body(int R, double* __restrict__ x, const float* __restrict__ e, Grid g)
{
    for (int i = g.b * blockDim.x + threadIdx.x; i < R; i += g.n * blockDim.x) x[i] += (double)e[i];
}

__device__ __forceinline__ void k_zero_f32_body(int R, float* __restrict__ v, Grid g)
{
    for (int i = g.b * blockDim.x + threadIdx.x; i < R; i += g.n * blockDim.x) v[i] = 0.0f;
}

// ---------------------------------------------------------------------------------------
// Nodal least-squares field
// ---------------------------------------------------------------------------------------
__device__ inline bool solve3(double M[3][3], double rhs[3], double sol[3])
{
    for (int piv = 0; piv < 3; ++piv) {
        int best = piv;
        for (int row = piv + 1; row < 3; ++row)
            if (fabs(M[row][piv]) > fabs(M[best][piv])) best = row;
        if (fabs(M[best][piv]) < 1.0e-18) return false;
        if (best != piv) {
            for (int c = 0; c < 3; ++c) {
                double t = M[best][c]; M[best][c] = M[piv][c]; M[piv][c] = t;
            }
            double t = rhs[best]; rhs[best] = rhs[piv]; rhs[piv] = t;
        }
        for (int row = piv + 1; row < 3; ++row) {
            double f = M[row][piv] / M[piv][piv];
            for (int c = piv; c < 3; ++c) M[row][c] -= f * M[piv][c];
            rhs[row] -= f * rhs[piv];
        }
    }
    for (int row = 2; row >= 0; --row) {
        double s = rhs[row];
        for (int c = row + 1; c < 3; ++c) s -= M[row][c] * sol[c];
        sol[row] = s / M[row][row];
    }
    return true;
}

// E of node i by the LSQ gradient; a separate function (not inlined) so that the single and
// the batched kernels run the same compiled arithmetic and agree bitwise.
static __device__ __noinline__ bool lsq_node(int64_t i, const double* __restrict__ xyz,
                                             const int32_t* __restrict__ gptr, const int32_t* __restrict__ gcol,
                                             const double* __restrict__ phi, double reg, double* __restrict__ E,
                                             float* __restrict__ Ef)
{
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, rhs[3] = {0, 0, 0}, sol[3] = {0, 0, 0};
    const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2], pi = phi[i];
    int cnt = 0;
    for (int e = gptr[i]; e < gptr[i + 1]; ++e) {
        int j = gcol[e];
        double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
        if (dx * dx + dy * dy + dz * dz <= 1e-24) continue;
        double dp = phi[j] - pi;
        M[0][0] += dx * dx; M[0][1] += dx * dy; M[0][2] += dx * dz;
        M[1][0] += dy * dx; M[1][1] += dy * dy; M[1][2] += dy * dz;
        M[2][0] += dz * dx; M[2][1] += dz * dy; M[2][2] += dz * dz;
        rhs[0] += dx * dp; rhs[1] += dy * dp; rhs[2] += dz * dp;
        ++cnt;
    }
    double ex = 0.0, ey = 0.0, ez = 0.0;
    if (cnt) {
        M[0][0] += reg; M[1][1] += reg; M[2][2] += reg;
        if (solve3(M, rhs, sol)) {
            ex = -sol[0]; ey = -sol[1]; ez = -sol[2];
        }
    }
    E[3 * i] = ex; E[3 * i + 1] = ey; E[3 * i + 2] = ez;
    if (Ef) {
        Ef[3 * i] = (float)ex; Ef[3 * i + 1] = (float)ey; Ef[3 * i + 2] = (float)ez;
    }
    return !(isfinite(ex) && isfinite(ey) && isfinite(ez));
}

__device__ __forceinline__ void k_lsq_field_body(int64_t N, const double* __restrict__ xyz, const int32_t* __restrict__ gptr,
                            const int32_t* __restrict__ gcol, const double* __restrict__ phi, double reg,
                            double* __restrict__ E, float* __restrict__ Ef, unsigned long long* flags, Grid g)
{
    bool bad = false;
    for (int64_t i = g.b * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)g.n * blockDim.x)
        bad = lsq_node(i, xyz, gptr, gcol, phi, reg, E, Ef) || bad;
    if (bad) atomicOr(flags, 1ull << 8);
}

// updateElectricField zeroes the whole field when any value is non-finite (PICCycle.cpp:883-893)
__device__ __forceinline__ void k_zero_if_flag_body(int64_t n3, double* E, float* Ef, const unsigned long long* flags, Grid g)
{
    if (!((*flags) & (1ull << 8))) return;
    for (int64_t i = g.b * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)g.n * blockDim.x) {
        E[i] = 0.0;
        if (Ef) Ef[i] = 0.0f;
    }
}


}  // namespace scdat
