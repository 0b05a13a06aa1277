// mg.cu -- lattice-multigrid preconditioned CG for the field solve (see mg.cuh).  Bandwidth
// kernels: every level's sweeps are CSR row loops (one thread per row, as the Jacobi-PCG SpMV),
// the transfers are the <= 8-entry rows of P and the <= 27-entry rows of P^T, the coarsest
// solve is a warp-per-row dense mat-vec held in L2.  FP32 (inner solve of the mixed form) or
// FP64 (the plain FP64 form).
#include "field_kern.cuh"
#include "mg.cuh"

namespace scdat {

namespace {

template <typename V> __device__ __forceinline__ const V* lv_val(const MgLevelDev& L);
template <> __device__ __forceinline__ const float* lv_val<float>(const MgLevelDev& L) { return L.valf; }
template <> __device__ __forceinline__ const double* lv_val<double>(const MgLevelDev& L) { return L.val; }
template <typename V> __device__ __forceinline__ const V* lv_diag(const MgLevelDev& L);
template <> __device__ __forceinline__ const float* lv_diag<float>(const MgLevelDev& L) { return L.diagf; }
template <> __device__ __forceinline__ const double* lv_diag<double>(const MgLevelDev& L) { return L.diag; }
template <typename V> __device__ __forceinline__ const V* lv_dinv(const MgLevelDev& L);
template <> __device__ __forceinline__ const float* lv_dinv<float>(const MgLevelDev& L) { return L.dinvf; }
template <> __device__ __forceinline__ const double* lv_dinv<double>(const MgLevelDev& L) { return L.dinv; }
template <typename V> __device__ __forceinline__ const V* pv_val(const PoissonView& A);
template <> __device__ __forceinline__ const float* pv_val<float>(const PoissonView& A) { return A.valf; }
template <> __device__ __forceinline__ const double* pv_val<double>(const PoissonView& A) { return A.val; }

// (A x)_i on a level
template <typename V>
__device__ __forceinline__ V lv_apply(const MgLevelDev& L, int i, const V* __restrict__ x)
{
    const V* val = lv_val<V>(L);
    V s = lv_diag<V>(L)[i] * x[i];
    for (int e = L.row_ptr[i]; e < L.row_ptr[i + 1]; ++e) s += val[e] * x[L.col[e]];
    return s;
}

}  // namespace

// x = omega D^-1 b (the first sweep from x = 0)
template <typename V>
__global__ void k_mg_smooth0(MgLevelDev L, const V* __restrict__ b, V* __restrict__ x, const PcgScalars* sc)
{
    if (sc->done) return;
    const V* dinv = lv_dinv<V>(L);
    const V om = (V)L.omega;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.R; i += gridDim.x * blockDim.x) x[i] = om * dinv[i] * b[i];
}

// xo = xi + omega D^-1 (b - A xi); with DOT, sc->rz = b . xo (the level-0 output z against r)
template <typename V, bool DOT>
__global__ void __launch_bounds__(256) k_mg_smooth(MgLevelDev L, const V* __restrict__ b, const V* __restrict__ xi,
                                                   V* __restrict__ xo, PcgScalars* sc, double* part)
{
    if (sc->done) return;
    const V* dinv = lv_dinv<V>(L);
    const V om = (V)L.omega;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.R; i += gridDim.x * blockDim.x) {
        const V bi = b[i];
        const V v = xi[i] + om * dinv[i] * (bi - lv_apply<V>(L, i, xi));
        xo[i] = v;
        if (DOT) acc[0] += (double)bi * (double)v;
    }
    if (DOT) {
        __shared__ double sh[32];
        block_sum<1>(acc, sh);
        if (last_block<1>(acc, part, &sc->ticket, Grid{blockIdx.x, gridDim.x})) sc->rz = acc[0];
    }
}

// res = b - A x
template <typename V>
__global__ void k_mg_residual(MgLevelDev L, const V* __restrict__ b, const V* __restrict__ x, V* __restrict__ res,
                              const PcgScalars* sc)
{
    if (sc->done) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.R; i += gridDim.x * blockDim.x)
        res[i] = b[i] - lv_apply<V>(L, i, x);
}

// bc = P^T res (L is the finer level, Rc the coarser level's rows)
template <typename V>
__global__ void k_mg_restrict(MgLevelDev L, int Rc, const V* __restrict__ res, V* __restrict__ bc, const PcgScalars* sc)
{
    if (sc->done) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < Rc; c += gridDim.x * blockDim.x) {
        V s = 0;
        for (int e = L.r_ptr[c]; e < L.r_ptr[c + 1]; ++e) s += (V)L.r_w[e] * res[L.r_col[e]];
        bc[c] = s;
    }
}

// xf += P xc
template <typename V>
__global__ void k_mg_prolong(MgLevelDev L, const V* __restrict__ xc, V* __restrict__ xf, const PcgScalars* sc)
{
    if (sc->done) return;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < L.R; f += gridDim.x * blockDim.x) {
        V s = 0;
        for (int e = L.p_ptr[f]; e < L.p_ptr[f + 1]; ++e) s += (V)L.p_w[e] * xc[L.p_col[e]];
        xf[f] += s;
    }
}

// x = Ainv b on the coarsest level: one warp per row, fixed-order lane sums
template <typename V>
__global__ void k_mg_coarse(int Rc, const V* __restrict__ inv, const V* __restrict__ b, V* __restrict__ x,
                            const PcgScalars* sc)
{
    if (sc->done) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < Rc; row += warps) {
        const V* a = inv + (size_t)row * Rc;
        V s = 0;
        for (int j = lane; j < Rc; j += 32) s += a[j] * b[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) x[row] = s;
    }
}

// ---- the CG on level 0 --------------------------------------------------------------------
template <typename V>
__global__ void __launch_bounds__(256) k_mgpcg_init(PoissonView A, const V* __restrict__ b, const V* __restrict__ x,
                                                    V* __restrict__ r, PcgScalars* sc, double* part)
{
    double acc[2] = {0.0, 0.0};
    const V* val = pv_val<V>(A);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.R; i += gridDim.x * blockDim.x) {
        const double ri = (double)b[i] - spmv_row(A, val, i, x);
        r[i] = (V)ri;
        acc[0] += ri * ri;
        acc[1] += (double)b[i] * (double)b[i];
    }
    __shared__ double sh[2 * 32];
    block_sum<2>(acc, sh);
    if (last_block<2>(acc, part, &sc->ticket, Grid{blockIdx.x, gridDim.x})) {
        sc->rr = acc[0];
        sc->bb = acc[1];
        sc->rz = 0.0;
        sc->rz_prev = 1.0;
        sc->iter = 0;
        double thr = sc->rtol * sc->rtol * (acc[1] > 0.0 ? acc[1] : 1.0);
        if (sc->abs_thr2 > 0.0) thr = sc->abs_thr2;
        sc->thr2 = thr;
        sc->done = (acc[0] <= thr || sc->max_iter <= 0) ? 1 : 0;
    }
}

template <typename V>
__global__ void k_mgpcg_dir(int R, const V* __restrict__ z, V* __restrict__ p, const PcgScalars* sc)
{
    if (sc->done) return;
    const bool first = sc->iter == 0;
    const V beta = first ? (V)0 : (V)(sc->rz / sc->rz_prev);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x)
        p[i] = first ? z[i] : z[i] + beta * p[i];
}

template <typename V>
__global__ void __launch_bounds__(256) k_mgpcg_spmv(PoissonView A, const V* __restrict__ p, V* __restrict__ q,
                                                    PcgScalars* sc, double* part)
{
    if (sc->done) return;
    const V* val = pv_val<V>(A);
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.R; i += gridDim.x * blockDim.x) {
        const double s = spmv_row(A, val, i, p);
        q[i] = (V)s;
        acc[0] += (double)p[i] * s;
    }
    __shared__ double sh[32];
    block_sum<1>(acc, sh);
    if (last_block<1>(acc, part, &sc->ticket, Grid{blockIdx.x, gridDim.x})) sc->pq = acc[0];
}

template <typename V>
__global__ void __launch_bounds__(256) k_mgpcg_update(int R, V* __restrict__ x, V* __restrict__ r,
                                                      const V* __restrict__ p, const V* __restrict__ q, PcgScalars* sc,
                                                      double* part)
{
    if (sc->done) return;
    const double pq = sc->pq;
    const double alpha = pq > 0.0 ? sc->rz / pq : 0.0;
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
        const double xi = (double)x[i] + alpha * (double)p[i];
        const double ri = (double)r[i] - alpha * (double)q[i];
        x[i] = (V)xi;
        r[i] = (V)ri;
        acc[0] += ri * ri;
    }
    __shared__ double sh[32];
    block_sum<1>(acc, sh);
    if (last_block<1>(acc, part, &sc->ticket, Grid{blockIdx.x, gridDim.x})) {
        sc->rz_prev = sc->rz;
        sc->rr = acc[0];
        sc->iter += 1;
        if (acc[0] <= sc->thr2 || sc->iter >= sc->max_iter || !(pq > 0.0)) sc->done = 1;
    }
}

// ---- launchers ------------------------------------------------------------------------------
namespace {

inline int blocks_for(int n, int gmax)
{
    const int b = (n + 255) / 256;
    return b < 1 ? 1 : (b > gmax ? gmax : b);
}

template <typename V>
void vcycle_level(const MgPlan& mg, int l, const V* b, V* out, PcgScalars* sc, double* part, cudaStream_t st)
{
    const MgLevelDev& L = mg.lv[l];
    const int g = blocks_for(L.R, mg.grid_max);
    if (l + 1 == (int)mg.lv.size()) {
        const V* inv;
        if constexpr (sizeof(V) == 4)
            inv = mg.cinvf;
        else
            inv = mg.cinv;
        k_mg_coarse<V><<<blocks_for(L.R * 32, mg.grid_max), 256, 0, st>>>(L.R, inv, b, out, sc);
        return;
    }
    const MgWork& w = mg.w[l];
    V* xa = static_cast<V*>(w.xa);
    V* xb = static_cast<V*>(w.xb);
    V* res = static_cast<V*>(w.res);
    const MgLevelDev& Cl = mg.lv[l + 1];
    V* bc = static_cast<V*>(mg.w[l + 1].b);
    V* xc = static_cast<V*>(mg.w[l + 1].xo);
    k_mg_smooth0<V><<<g, 256, 0, st>>>(L, b, xa, sc);
    k_mg_smooth<V, false><<<g, 256, 0, st>>>(L, b, xa, xb, sc, part);
    k_mg_residual<V><<<g, 256, 0, st>>>(L, b, xb, res, sc);
    k_mg_restrict<V><<<blocks_for(Cl.R, mg.grid_max), 256, 0, st>>>(L, Cl.R, res, bc, sc);
    vcycle_level<V>(mg, l + 1, bc, xc, sc, part, st);
    k_mg_prolong<V><<<g, 256, 0, st>>>(L, xc, xb, sc);
    k_mg_smooth<V, false><<<g, 256, 0, st>>>(L, b, xb, xa, sc, part);
    if (l == 0)
        k_mg_smooth<V, true><<<g, 256, 0, st>>>(L, b, xa, out, sc, part);
    else
        k_mg_smooth<V, false><<<g, 256, 0, st>>>(L, b, xa, out, sc, part);
}

}  // namespace

template <typename V>
void launch_vcycle(const MgPlan& mg, const V* r, V* z, PcgScalars* sc, double* part, cudaStream_t st)
{
    vcycle_level<V>(mg, 0, r, z, sc, part, st);
}

template <typename V>
void launch_mgpcg_init(const PoissonView& A, const V* b, const V* x, V* r, PcgScalars* sc, double* part, int grid,
                       cudaStream_t st)
{
    k_mgpcg_init<V><<<grid, 256, 0, st>>>(A, b, x, r, sc, part);
}

template <typename V>
void launch_mgpcg_iter(const PoissonView& A, const MgPlan& mg, V* x, V* r, V* z, V* p, V* q, PcgScalars* sc,
                       double* part, int grid, cudaStream_t st)
{
    k_mgpcg_dir<V><<<grid, 256, 0, st>>>(A.R, z, p, sc);
    k_mgpcg_spmv<V><<<grid, 256, 0, st>>>(A, p, q, sc, part);
    k_mgpcg_update<V><<<grid, 256, 0, st>>>(A.R, x, r, p, q, sc, part);
    launch_vcycle<V>(mg, r, z, sc, part, st);
}

template void launch_vcycle<float>(const MgPlan&, const float*, float*, PcgScalars*, double*, cudaStream_t);
template void launch_vcycle<double>(const MgPlan&, const double*, double*, PcgScalars*, double*, cudaStream_t);
template void launch_mgpcg_init<float>(const PoissonView&, const float*, const float*, float*, PcgScalars*, double*,
                                       int, cudaStream_t);
template void launch_mgpcg_init<double>(const PoissonView&, const double*, const double*, double*, PcgScalars*,
                                        double*, int, cudaStream_t);
template void launch_mgpcg_iter<float>(const PoissonView&, const MgPlan&, float*, float*, float*, float*, float*,
                                       PcgScalars*, double*, int, cudaStream_t);
template void launch_mgpcg_iter<double>(const PoissonView&, const MgPlan&, double*, double*, double*, double*,
                                        double*, PcgScalars*, double*, int, cudaStream_t);

}  // namespace scdat
