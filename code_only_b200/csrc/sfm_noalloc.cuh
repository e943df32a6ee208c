// sfm_noalloc.cuh -- a uniform periodic base-grid solve that allocates
// nothing (exported as sfm_uniform_solve_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a
// solve: code running inside a fixed memory pool or an arena handed out at
// start-up, a real-time step whose allocator calls would synchronise the
// device, or a host library that has promised its user a fixed device
// footprint.  For them this entry point runs the base-grid multigrid of
// sfm_mg.cuh (mg_lin as repeated defect corrections, mg.F90:42-94) on the
// caller's device buffers, with every working array in one file-scope
// __device__ array of fixed size.  Nothing is allocated: no cudaMalloc, no
// cudaFree, no allocating library call.  The only set-up is the lookup of
// that array's device address, once per device (cudaGetSymbolAddress).
//
// Limits and contract:
//   - n (cells per edge) is a power of two, 2 <= n <= SFM_NOALLOC_MAX_N (32);
//     the scratch holds the level arrays for n = 32, about 2 MiB;
//   - the kernel clears every scratch array it reads before its first read,
//     so the scratch needs no zeroing by the caller and no state carries
//     over from one call to the next;
//   - there is one scratch array per device and loaded library: two calls on
//     the same device whose executions overlap (different streams without an
//     ordering between them, or different host threads) race on it and give
//     wrong results.  Order such calls on one stream or with events;
//   - the first call on each device does the set-up lookup; make that first
//     call before any stream capture on that device.
#pragma once
#include "sfm_mg.cuh"

namespace sfm {

constexpr int NOALLOC_MAX_N = 32;

// doubles of the U/RES/RHS/RHO arrays of every level of an n^3 base grid,
// plus SRC and PSI on level 0
__host__ __device__ constexpr size_t noalloc_level_doubles(int n) {
    size_t tot = 0;
    for (int m = 0; (n >> m) >= 1; m++) {
        const size_t G = (size_t)(n >> m) + 2;
        tot += 4 * G * G * G;
    }
    const size_t G0 = (size_t)n + 2;
    return tot + 2 * G0 * G0 * G0;
}
// two result words follow the arrays: relative residual and cycle count
constexpr size_t NOALLOC_OUT_DOUBLES = 2;
constexpr size_t NOALLOC_SCRATCH_DOUBLES = noalloc_level_doubles(NOALLOC_MAX_N) + NOALLOC_OUT_DOUBLES;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// level arrays of an n^3 base grid laid out from the start of the scratch
__host__ __device__ inline MgData noalloc_layout(double *s, int n, double h) {
    MgData d;
    for (int m = 0; m < MG_MAXLEV; m++) d.U[m] = d.RES[m] = d.RHS[m] = d.RHO[m] = nullptr;
    int MMax = 0;
    while ((1 << MMax) < n) MMax++;
    for (int m = 0; m <= MMax; m++) {
        const size_t G = (size_t)(n >> m) + 2, V = G * G * G;
        d.U[m] = s; s += V;
        d.RES[m] = s; s += V;
        d.RHS[m] = s; s += V;
        d.RHO[m] = s; s += V;
    }
    const size_t G0 = (size_t)n + 2, V0 = G0 * G0 * G0;
    d.SRC = s; s += V0;
    d.PSI = s;
    d.N = n;
    d.MMax = MMax;
    d.hbase = h;
    d.periodic = 1;
    d.zbc = 0;
    for (int f = 0; f < 6; f++) d.touch[f] = 0;   // periodic: no face touches a physical boundary
    return d;
}

// One CTA.  rho and psi are dense n^3 arrays, x fastest.  Solves
// lap(psi) = four_pi_G * (rho - mean rho) on the periodic grid of cell width
// h: psi starts at zero; each cycle forms the residual (mg_poisson.F90:5-28),
// solves for the correction with mg_lin and adds it (mg.F90:62-90), until
// max|residual| <= rel_tol * max|four_pi_G (rho - mean)| or max_cycles.
__global__ void __launch_bounds__(1024) k_mg_uniform_noalloc(MgData d, const double *__restrict__ rho,
                                                             double *__restrict__ psi, double four_pi_G,
                                                             double rel_tol, int max_cycles, double *out,
                                                             int64_t clear_doubles) {
    __shared__ double sh[32];
    __shared__ double wsum[32];
    const int n = d.N, G = n + 2, n3 = n * n * n;
    // one CTA, every level in the scratch array (global memory)
    MgRun r;
    r.rank = 0;
    r.nct = 1;
    r.wide_min = 1 << 30;
    r.smem_from = d.MMax + 1;
    r.pending = false;
    r.mirror = nullptr;
    r.slot = nullptr;
    // every array read below starts at zero (U, RES, RHS, RHO of all levels, SRC, PSI)
    for (int64_t t = threadIdx.x; t < clear_doubles; t += blockDim.x) d.U[0][t] = 0.0;
    // A NaN or Inf density would make the mean and every source value NaN;
    // max|source| would then stay 0 (NaN fails every comparison) and the
    // loop would stop at once with psi = 0 reported as converged.  Refuse
    // it instead: psi is set to NaN everywhere and the result words carry a
    // cycle count of -1, which the host turns into SFM_ENONFINITE.
    int bad = 0;
    for (int c = threadIdx.x; c < n3; c += blockDim.x) bad |= !isfinite(rho[c]);
    if (__syncthreads_or(bad)) {
        for (int c = threadIdx.x; c < n3; c += blockDim.x) psi[c] = __longlong_as_double(0x7ff8000000000000LL);
        if (threadIdx.x == 0) {
            out[0] = __longlong_as_double(0x7ff8000000000000LL);
            out[1] = -1.0;
        }
        return;
    }
    // mean of rho: per-thread sums in cell order, then a fixed tree (deterministic)
    double s = 0.0;
    for (int c = threadIdx.x; c < n3; c += blockDim.x) s = s + rho[c];
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot = tot + wsum[w];
    const double mean = tot / (double)n3;
    double smax = 0.0;
    for (int c = threadIdx.x; c < n3; c += blockDim.x) {
        const double v = four_pi_G * (rho[c] - mean);
        d.SRC[cidx(G, c % n, (c / n) % n, c / (n * n))] = v;
        const double a = fabs(v);
        smax = a > smax ? a : smax;
    }
    smax = mg_block_max(smax, sh);   // synchronises the CTA
    int it = 0;
    double rrel = 0.0;
    for (;;) {
        mg_resid(r, d, 0, d.RHO[0], d.PSI, d.SRC);
        double v = 0.0;
        for (int c = threadIdx.x; c < n3; c += blockDim.x) {
            const double a = fabs(d.RHO[0][cidx(G, c % n, (c / n) % n, c / (n * n))]);
            v = a > v ? a : v;
        }
        const double rmax = mg_block_max(v, sh);
        rrel = smax > 0.0 ? rmax / smax : 0.0;
        if (rrel <= rel_tol || it >= max_cycles) break;
        mg_lin(r, d, sh);
        mg_addw(r, d, 0, d.PSI, d.U[0]);
        it++;
    }
    for (int c = threadIdx.x; c < n3; c += blockDim.x) psi[c] = d.PSI[cidx(G, c % n, (c / n) % n, c / (n * n))];
    if (threadIdx.x == 0) {
        out[0] = rrel;
        out[1] = (double)it;
    }
}

}  // namespace sfm
