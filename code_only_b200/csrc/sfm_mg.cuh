// sfm_mg.cuh -- the uniform base-grid multigrid (mg.F90, mg_poisson.F90,
// mg_interpol_cubic.F90) as one persistent CTA.
//
// The reference gathers the base level to rank 0 and runs mg_cycle there
// serially (vmg.F90:407-428, mg_data.F90:179-330).  Here the whole cycle
// (<= 10 defect corrections of an FMG with Ncycle 2, 2/2 smoothing) runs in
// one CTA of 512 threads on a base grid of at most 64^3 cells: the coarse
// levels' working arrays in shared memory, level 0 and the data exchanged
// with the AMR levels in global memory (L2), every operation separated by
// __syncthreads; nothing returns to the host.  FP64 throughout (the
// coarsest-level solve stays in FP64 in the mixed-precision path).
#pragma once
#include "sfm_device.cuh"

namespace sfm {

constexpr int MG_MAXLEV = 8;
constexpr int MG_NMAX = 128;   // base-grid cells per edge (the mg CTA handles at most 64)

struct MgData {
    double *U[MG_MAXLEV], *RES[MG_MAXLEV], *RHS[MG_MAXLEV], *RHO[MG_MAXLEV];
    double *SRC, *PSI;   // level 0 only
    int N;               // cells per edge on level 0
    int MMax;            // coarsest level (1 cell)
    double hbase;        // cell width on level 0 (fmg_get_h(Lmin, FMG_LevelMax))
    int periodic;        // mg_boundary_u wraps (periodic module) or is a no-op (sphere)
    int touch[6];        // TouchBoundary of the base grid (mg_data.F90:77-83)
};

__device__ __forceinline__ int mgN(const MgData &d, int m) { return d.N >> m; }
// cell (i, j, k) of flat index c in an n^3 level, n a power of two (ln = log2 n):
// shifts and masks instead of integer division
__device__ __forceinline__ void mg_ijk(int c, int n, int ln, int &i, int &j, int &k) {
    i = c & (n - 1);
    j = (c >> ln) & (n - 1);
    k = c >> (2 * ln);
}
__device__ __forceinline__ double mgH(const MgData &d, int m) { return d.hbase * (double)(1 << m); }

__device__ double mg_block_max(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) {
        double t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = sh[w] > m ? sh[w] : m;
    __syncthreads();
    return m;
}

// (p, q) = (t mod G, t div G) for t < G^2 <= 130^2 without an integer
// division: (t + 1/2) / G lies at least 1/(2G) from an integer, far above
// the float rounding of (t + 1/2) * (1/G)
__device__ __forceinline__ void mg_pq(int t, int G, float rG, int &p, int &q) {
    q = (int)(((float)t + 0.5f) * rG);
    p = t - q * G;
}
// periodic wrap of one ghost layer (fmg_boundary_phys_periodic.F90:71-104).
// The reference copies x, then y, then z faces, each face including the
// ghost rows of the other directions; after the three passes every ghost
// cell holds the interior cell at its periodic image (wrap each coordinate
// -1 -> n-1, n -> 0).  That final state is written here in one pass:
// cells on several faces are written with the same value more than once.
__device__ void mg_boundary_u(const MgData &d, int m, double *a) {
    if (!d.periodic) return;
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    auto wrap = [n](int x) { return x < 0 ? n - 1 : (x >= n ? 0 : x); };
    for (int t = threadIdx.x; t < 3 * G * G; t += blockDim.x) {
        const int dir = t >= 2 * G * G ? 2 : (t >= G * G ? 1 : 0);
        int p, q, i, j, k;
        mg_pq(t - dir * G * G, G, rG, p, q);
        put3(dir, -1, p - 1, q - 1, i, j, k);
        a[cidx(G, i, j, k)] = a[cidx(G, wrap(i), wrap(j), wrap(k))];
        put3(dir, n, p - 1, q - 1, i, j, k);
        a[cidx(G, i, j, k)] = a[cidx(G, wrap(i), wrap(j), wrap(k))];
    }
    __syncthreads();
}
__device__ void mg_boundary_fill0(const MgData &d, int m, double *a) {   // mg.F90:735-750
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    for (int f = 0; f < 6; f++) {
        if (!d.touch[f]) continue;
        for (int t = threadIdx.x; t < G * G; t += blockDim.x) {
            int i, j, k, p, q;
            mg_pq(t, G, rG, p, q);
            put3(f >> 1, (f & 1) ? n : -1, p - 1, q - 1, i, j, k);
            a[cidx(G, i, j, k)] = 0.0;
        }
    }
    __syncthreads();
}
__device__ void mg_boundary_extrap(const MgData &d, int m, double *a) {  // mg.F90:754-771
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    for (int dir = 0; dir < 3; dir++) {
        for (int lr = 0; lr < 2; lr++) {
            if (!d.touch[lr + 2 * dir]) continue;
            for (int t = threadIdx.x; t < G * G; t += blockDim.x) {
                int i, j, k, ii, jj, kk, p, q;
                mg_pq(t, G, rG, p, q);
                put3(dir, lr ? n : -1, p - 1, q - 1, i, j, k);
                put3(dir, lr ? n - 1 : 0, p - 1, q - 1, ii, jj, kk);
                a[cidx(G, i, j, k)] = -a[cidx(G, ii, jj, kk)];
            }
        }
        __syncthreads();
    }
}
__device__ __forceinline__ double mg_lap_sum(const double *u, int G, int i, int j, int k) {
    double s = u[cidx(G, i + 1, j, k)] + u[cidx(G, i - 1, j, k)];
    s = s + u[cidx(G, i, j + 1, k)];
    s = s + u[cidx(G, i, j - 1, k)];
    s = s + u[cidx(G, i, j, k + 1)];
    s = s + u[cidx(G, i, j, k - 1)];
    s = s - 6.0 * u[cidx(G, i, j, k)];
    return s;
}
__device__ void mg_resid(const MgData &d, int m, double *res, double *u, const double *rhs) {   // mg_poisson.F90:5-28
    const int n = mgN(d, m), G = n + 2, ln = __ffs(n) - 1;
    double hh = mgH(d, m);
    double h2i = 1.0 / (hh * hh);
    mg_boundary_u(d, m, u);
    for (int c = threadIdx.x; c < n * n * n; c += blockDim.x) {
        int i, j, k;
        mg_ijk(c, n, ln, i, j, k);
        res[cidx(G, i, j, k)] = -h2i * mg_lap_sum(u, G, i, j, k) + rhs[cidx(G, i, j, k)];
    }
    __syncthreads();
}
// both colours (mg_poisson.F90:32-79); returns this thread's max|resh2|:
// Resmaxg = (max over the CTA) / h^2 is formed by the caller where it is
// used (the max is exact, so where it is reduced does not change it)
__device__ double mg_relax(const MgData &d, int m, double *u, const double *rhs) {
    const int n = mgN(d, m), G = n + 2;
    double hh = mgH(d, m), h2 = hh * hh, rm = 0.0;
    const int half = (n * n * n + 1) / 2;
    (void)G;
    for (int ipass = 1; ipass <= 2; ipass++) {
        mg_boundary_u(d, m, u);
        for (int c = threadIdx.x; c < half; c += blockDim.x) {
            int i2, j, k, i;
            if (n == 1) { if (((ipass) & 1) != 0) continue; i = 0; j = 0; k = 0; }
            else {
                int hn = n / 2;
                const int lhn = __ffs(hn) - 1;
                i2 = c & (hn - 1); j = (c >> lhn) & (n - 1); k = c >> (lhn + __ffs(n) - 1);
                i = 2 * i2 + ((j + k + ipass) & 1);
            }
            double resh2 = mg_lap_sum(u, G, i, j, k) - h2 * rhs[cidx(G, i, j, k)];
            u[cidx(G, i, j, k)] = u[cidx(G, i, j, k)] + (1.0 / 6.0) * resh2;
            double a = fabs(resh2);
            rm = a > rm ? a : rm;
        }
        __syncthreads();
    }
    return rm;
}
__device__ void mg_rstrct(const MgData &d, int m, double *uc, const double *uf) {   // linear (mg.F90:581-602)
    const int n = mgN(d, m), G = n + 2, Gf = 2 * n + 2, ln = __ffs(n) - 1;
    for (int c = threadIdx.x; c < n * n * n; c += blockDim.x) {
        int i, j, k;
        mg_ijk(c, n, ln, i, j, k);
        uc[cidx(G, i, j, k)] = rstrct_linear(uf, Gf, 2 * i, 2 * j, 2 * k);
    }
    __syncthreads();
}
__device__ void mg_interp(const MgData &d, int m, double *uf, double *uc, bool cubic) {   // mg.F90:608-633
    const int lc = m + 1, n = mgN(d, m), G = n + 2, nc = mgN(d, lc), Gc = nc + 2, ln = __ffs(n) - 1;
    // Lagrange nodes and weights per fine index, evaluated once per call
    __shared__ int tcw[MG_NMAX][4];
    __shared__ double tww[MG_NMAX][4];
    const bool tri = cubic && nc + 2 >= 4;
    if (tri && (int)threadIdx.x < n) cubic_weights((int)threadIdx.x, -1, nc, tcw[threadIdx.x], tww[threadIdx.x]);
    mg_boundary_extrap(d, lc, uc);   // ends with __syncthreads
    mg_boundary_u(d, lc, uc);
    for (int c = threadIdx.x; c < n * n * n; c += blockDim.x) {
        int i, j, k;
        mg_ijk(c, n, ln, i, j, k);
        uf[cidx(G, i, j, k)] = tri ? tricubic_cell_w(uc, Gc, tcw[i], tww[i], tcw[j], tww[j], tcw[k], tww[k])
                                   : trilinear_cell(uc, Gc, i, j, k, 0, 0, 0);
    }
    __syncthreads();
    mg_boundary_fill0(d, m, uf);
    mg_boundary_fill0(d, lc, uc);
    mg_boundary_u(d, m, uf);
    mg_boundary_u(d, lc, uc);
}
__device__ void mg_fill0(const MgData &d, int m, double *a) {
    const int G = mgN(d, m) + 2;
    for (int c = threadIdx.x; c < G * G * G; c += blockDim.x) a[c] = 0.0;
    __syncthreads();
}
__device__ void mg_copy(const MgData &d, int m, double *o, const double *a) {
    const int G = mgN(d, m) + 2;
    for (int c = threadIdx.x; c < G * G * G; c += blockDim.x) o[c] = a[c];
    __syncthreads();
}
__device__ void mg_addw(const MgData &d, int m, double *a, const double *da) {
    const int G = mgN(d, m) + 2;
    for (int c = threadIdx.x; c < G * G * G; c += blockDim.x) a[c] = a[c] + da[c];
    __syncthreads();
}

// mg_lin (mg.F90:106-218); returns the last Resmaxg (the Resmaxg of every
// earlier mg_relax is overwritten unread, so only the last one is reduced)
__device__ double mg_lin(const MgData &d, double *sh) {
    double rm = 0.0;   // this thread's max|resh2| of the last mg_relax
    int mr = d.MMax;   // its level
    for (int m = 1; m <= d.MMax; m++) mg_rstrct(d, m, d.RHO[m], d.RHO[m - 1]);
    mg_fill0(d, d.MMax, d.U[d.MMax]);
    for (int q = 0; q < 2; q++) rm = mg_relax(d, d.MMax, d.U[d.MMax], d.RHO[d.MMax]);
    for (int m = d.MMax - 1; m >= 0; m--) {
        mg_interp(d, m, d.U[m], d.U[m + 1], true);
        mg_copy(d, m, d.RHS[m], d.RHO[m]);
        for (int jc = 1; jc <= 2; jc++) {
            for (int v = m; v <= d.MMax - 1; v++) {
                for (int q = 0; q < 2; q++) rm = mg_relax(d, v, d.U[v], d.RHS[v]);
                mr = v;
                mg_resid(d, v, d.RES[v], d.U[v], d.RHS[v]);
                mg_rstrct(d, v + 1, d.RHS[v + 1], d.RES[v]);
                mg_fill0(d, v + 1, d.U[v + 1]);
            }
            for (int q = 0; q < 2; q++) rm = mg_relax(d, d.MMax, d.U[d.MMax], d.RHS[d.MMax]);
            mr = d.MMax;
            for (int v = d.MMax - 1; v >= m; v--) {
                mg_interp(d, v, d.RES[v], d.U[v + 1], false);
                mg_addw(d, v, d.U[v], d.RES[v]);
                for (int q = 0; q < 2; q++) rm = mg_relax(d, v, d.U[v], d.RHS[v]);
                mr = v;
            }
        }
    }
    const double hh = mgH(d, mr);
    return mg_block_max(rm, sh) / (hh * hh);
}

// dynamic shared memory of the base-grid CTA
__device__ __forceinline__ double *mg_dyn_smem() {
    extern __shared__ double mg_smem[];
    return mg_smem;
}

// Shared-memory plan: U, RES and RHS of the coarse levels m >= smem_from
// (smem_from >= 1) live in shared memory (their values never carry over
// between calls: mg_lin rewrites every cell it reads, mg.F90:142-215);
// level 0's arrays, PSI, SRC and RHO stay in global memory.  Level 0 is
// never placed in shared memory: with it there, the B200 build read stale
// level-0 values and the base solve lost bitwise parity (levels >= 1 in
// shared memory are bit-identical to the all-global layout).
__host__ __device__ inline int mg_smem_from(int N, int MMax, size_t budget_doubles, size_t *used) {
    size_t tot = 0;
    int from = MMax + 1;
    for (int m = MMax; m >= 1; m--) {
        size_t G = (size_t)(N >> m) + 2, V = G * G * G;
        if (tot + 3 * V > budget_doubles) break;
        tot += 3 * V;
        from = m;
    }
    if (used) *used = tot;
    return from;
}

// mg_cycle (mg.F90:42-94) with ju = PSI, jrho = SRC; one CTA
// (nmax: cap on the defect corrections, 10 in the reference)
__global__ void __launch_bounds__(512, 1) k_mg_cycle(MgData dg, int smem_from, int *iters_out, int nmax) {
    pdl_enter();
    __shared__ double sh[32];
    MgData d = dg;
    {
        double *p = mg_dyn_smem();
        for (int m = d.MMax; m >= smem_from; m--) {
            size_t G = (size_t)(d.N >> m) + 2, V = G * G * G;
            d.U[m] = p; p += V;
            d.RES[m] = p; p += V;
            d.RHS[m] = p; p += V;
        }
        const int64_t tot = p - mg_dyn_smem();
        double *z = mg_dyn_smem();
        for (int64_t t = threadIdx.x; t < tot; t += blockDim.x) z[t] = 0.0;
        __syncthreads();
    }
    const double errmax = (double)1.e-2f;   // default-real literal (mg.F90:50)
    mg_boundary_fill0(d, 0, d.PSI);
    mg_boundary_u(d, 0, d.PSI);
    double rhomax = 0.0;
    int it;
    for (it = 1; it <= nmax; it++) {
        mg_resid(d, 0, d.RHO[0], d.PSI, d.SRC);
        if (it == 1) {
            const int n = d.N, G = n + 2;
            double v = 0.0;
            for (int c = threadIdx.x; c < n * n * n; c += blockDim.x) {
                int i, j, k;
                mg_ijk(c, n, __ffs(n) - 1, i, j, k);
                double a = fabs(d.RHO[0][cidx(G, i, j, k)]);
                v = a > v ? a : v;
            }
            rhomax = mg_block_max(v, sh);
        }
        double res = mg_lin(d, sh);
        mg_addw(d, 0, d.PSI, d.U[0]);
        if (res / rhomax < errmax) break;
    }
    if (threadIdx.x == 0 && iters_out) *iters_out = it > nmax ? nmax : it;
}

}  // namespace sfm
