// sfm_mg.cuh -- the uniform base-grid multigrid (mg.F90, mg_poisson.F90,
// mg_interpol_cubic.F90) as one persistent CTA or one thread-block cluster.
//
// The reference gathers the base level to rank 0 and runs mg_cycle there
// serially (vmg.F90:407-428, mg_data.F90:179-330).  Here the whole cycle
// (<= 10 defect corrections of an FMG with Ncycle 2, 2/2 smoothing) runs in
// one launch of 512-thread CTAs on a base grid of at most 64^3 cells: the
// coarse levels' working arrays in shared memory, the large levels and the
// data exchanged with the AMR levels in global memory (L2), every operation
// separated by a CTA or cluster barrier; nothing returns to the host.  FP64
// throughout (the coarsest-level solve stays in FP64 in the mixed-precision
// path).
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
    int zbc;             // mg_boundary_u on the z faces: 1 mirrors the z-min face
                         // (zmirror module), 2 wraps z (the z-periodic cylinders)
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

// ---------------------------------------------------------------------------
// One CTA or a thread-block cluster.  With a cluster, the steps on the large
// levels (at least wide_min cells per edge; their arrays in global memory,
// L2-resident) are spread over every thread of every CTA and end with a
// cluster barrier; the steps on the small levels run on CTA 0 alone, their
// arrays in its shared memory, separated by __syncthreads, while the other
// CTAs skip them and wait at the next large-level step.  Each cell is still
// computed by one thread with the same expression, and the maxima are exact,
// so the result does not depend on the CTA count.  Distributed shared memory
// is read twice: the cluster-wide maximum (one value per CTA), and the copy
// of a small level into every CTA before it is interpolated onto a large one.
// ---------------------------------------------------------------------------
struct MgRun {
    int rank, nct;     // this CTA's rank in the cluster, CTAs in the cluster (1: one CTA)
    int wide_min;      // levels with at least this many cells per edge use the whole cluster
    int smem_from;     // first level whose U / RES / RHS live in CTA 0's shared memory
    bool pending;      // a step ran on CTA 0 alone since the last cluster barrier
    double *mirror;    // this CTA's copy of a small level (interpolation onto a large level)
    double *slot;      // this CTA's contribution to a cluster-wide maximum
};
struct MgStep {
    int start, stride; // this thread's first cell index and the step between its cells
    bool on;           // this CTA works on the step
    bool wide;         // the step uses the whole cluster
};
__device__ __forceinline__ void mg_cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// generic address of the same shared-memory variable in CTA `rank` of the cluster
__device__ __forceinline__ double *mg_map_rank(double *p, int rank) {
    uint64_t out;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"(p), "r"(rank));
    return reinterpret_cast<double *>(out);
}
__device__ __forceinline__ bool mg_wide(const MgRun &r, const MgData &d, int m) {
    return r.nct > 1 && (d.N >> m) >= r.wide_min;
}
// start of a step on level m: a large-level step first waits (cluster
// barrier) for whatever CTA 0 did alone before it
__device__ __forceinline__ MgStep mg_begin(MgRun &r, const MgData &d, int m) {
    MgStep s;
    s.wide = mg_wide(r, d, m);
    if (s.wide) {
        if (r.pending) {
            mg_cluster_sync();
            r.pending = false;
        }
        s.start = r.rank * (int)blockDim.x + (int)threadIdx.x;
        s.stride = r.nct * (int)blockDim.x;
        s.on = true;
    } else {
        r.pending = r.nct > 1;
        s.start = (int)threadIdx.x;
        s.stride = (int)blockDim.x;
        s.on = r.rank == 0;
    }
    return s;
}
__device__ __forceinline__ void mg_end(const MgStep &s) {
    if (s.wide) mg_cluster_sync();
    else if (s.on) __syncthreads();
}

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

// maximum over the CTA, and over the cluster when the step is a large-level
// one (every CTA's value through distributed shared memory); all threads of
// every working CTA get the result
__device__ double mg_max(MgRun &r, double v, double *sh, bool wide) {
    const double m = mg_block_max(v, sh);
    if (!wide) return m;
    if (threadIdx.x == 0) *r.slot = m;
    mg_cluster_sync();
    double g = 0.0;
    for (int q = 0; q < r.nct; q++) {
        const double t = *mg_map_rank(r.slot, q);
        g = t > g ? t : g;
    }
    mg_cluster_sync();   // no CTA overwrites its slot while another may still read it
    return g;
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
__device__ void mg_boundary_u(MgRun &r, const MgData &d, int m, double *a) {
    if (d.zbc == 1) {   // u(:,:,-1) = u(:,:,0) (fmg_boundary_phys_zmirror.F90:84-96)
        const int n = mgN(d, m), G = n + 2;
        const MgStep s = mg_begin(r, d, m);
        if (s.on)
            for (int t = s.start; t < G * G; t += s.stride) a[(int64_t)t] = a[(int64_t)t + G * G];
        mg_end(s);
        return;
    }
    if (d.zbc == 2) {   // u(:,:,-1) = u(:,:,n-1), then u(:,:,n) = u(:,:,0) (cyl_zperiodic.F90:60-72)
        const int n = mgN(d, m), G = n + 2;
        const int64_t P = (int64_t)G * G;
        MgStep s = mg_begin(r, d, m);
        if (s.on)
            for (int t = s.start; t < G * G; t += s.stride) a[t] = a[t + n * P];
        mg_end(s);
        s = mg_begin(r, d, m);
        if (s.on)
            for (int t = s.start; t < G * G; t += s.stride) a[t + (n + 1) * P] = a[t + P];
        mg_end(s);
        return;
    }
    if (!d.periodic) return;
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    auto wrap = [n](int x) { return x < 0 ? n - 1 : (x >= n ? 0 : x); };
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int t = s.start; t < 3 * G * G; t += s.stride) {
            const int dir = t >= 2 * G * G ? 2 : (t >= G * G ? 1 : 0);
            int p, q, i, j, k;
            mg_pq(t - dir * G * G, G, rG, p, q);
            put3(dir, -1, p - 1, q - 1, i, j, k);
            a[cidx(G, i, j, k)] = a[cidx(G, wrap(i), wrap(j), wrap(k))];
            put3(dir, n, p - 1, q - 1, i, j, k);
            a[cidx(G, i, j, k)] = a[cidx(G, wrap(i), wrap(j), wrap(k))];
        }
    mg_end(s);
}
// A step with nothing to do (no face of the box on the physical boundary:
// a periodic box) is skipped with its barrier: the previous step's barrier
// already orders what came before it against what follows.
__device__ __forceinline__ bool mg_touches(const MgData &d, int f0, int f1) {
    bool t = false;
    for (int f = f0; f < f1; f++) t = t || d.touch[f];
    return t;
}
__device__ void mg_boundary_fill0(MgRun &r, const MgData &d, int m, double *a) {   // mg.F90:735-750
    if (!mg_touches(d, 0, 6)) return;
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int f = 0; f < 6; f++) {
            if (!d.touch[f]) continue;
            for (int t = s.start; t < G * G; t += s.stride) {
                int i, j, k, p, q;
                mg_pq(t, G, rG, p, q);
                put3(f >> 1, (f & 1) ? n : -1, p - 1, q - 1, i, j, k);
                a[cidx(G, i, j, k)] = 0.0;
            }
        }
    mg_end(s);
}
__device__ void mg_boundary_extrap(MgRun &r, const MgData &d, int m, double *a) {  // mg.F90:754-771
    const int n = mgN(d, m), G = n + 2;
    const float rG = 1.0f / (float)G;
    for (int dir = 0; dir < 3; dir++) {
        if (!mg_touches(d, 2 * dir, 2 * dir + 2)) continue;
        const MgStep s = mg_begin(r, d, m);
        if (s.on)
            for (int lr = 0; lr < 2; lr++) {
                if (!d.touch[lr + 2 * dir]) continue;
                for (int t = s.start; t < G * G; t += s.stride) {
                    int i, j, k, ii, jj, kk, p, q;
                    mg_pq(t, G, rG, p, q);
                    put3(dir, lr ? n : -1, p - 1, q - 1, i, j, k);
                    put3(dir, lr ? n - 1 : 0, p - 1, q - 1, ii, jj, kk);
                    a[cidx(G, i, j, k)] = -a[cidx(G, ii, jj, kk)];
                }
            }
        mg_end(s);
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
// The same sum on a periodic box, each neighbour read at its periodic image
// instead of from the ghost layer: the values a wrap of the ghost layer
// (mg_boundary_u) would have put there, so the sum is the same to the bit.
// The relaxation and the residual read only these six face neighbours, so
// on periodic boxes they skip the wrap step (and its barrier) the reference
// does before each of them; their u ghost layers are then left as they
// were, and every reader of ghost cells (the prolongation, which also reads
// edges and corners) wraps its level itself first.
__device__ __forceinline__ double mg_lap_sum_wrap(const double *u, int G, int n, int i, int j, int k) {
    const int ip = i + 1 == n ? 0 : i + 1, im = i == 0 ? n - 1 : i - 1;
    const int jp = j + 1 == n ? 0 : j + 1, jm = j == 0 ? n - 1 : j - 1;
    const int kp = k + 1 == n ? 0 : k + 1, km = k == 0 ? n - 1 : k - 1;
    double s = u[cidx(G, ip, j, k)] + u[cidx(G, im, j, k)];
    s = s + u[cidx(G, i, jp, k)];
    s = s + u[cidx(G, i, jm, k)];
    s = s + u[cidx(G, i, j, kp)];
    s = s + u[cidx(G, i, j, km)];
    s = s - 6.0 * u[cidx(G, i, j, k)];
    return s;
}
__device__ void mg_resid(MgRun &r, const MgData &d, int m, double *res, double *u, const double *rhs) {   // mg_poisson.F90:5-28
    const int n = mgN(d, m), G = n + 2, ln = __ffs(n) - 1;
    double hh = mgH(d, m);
    double h2i = 1.0 / (hh * hh);
    if (d.zbc) mg_boundary_u(r, d, m, u);   // mg_poisson.F90:16
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int c = s.start; c < n * n * n; c += s.stride) {
            int i, j, k;
            mg_ijk(c, n, ln, i, j, k);
            const double lap = d.periodic ? mg_lap_sum_wrap(u, G, n, i, j, k) : mg_lap_sum(u, G, i, j, k);
            res[cidx(G, i, j, k)] = -h2i * lap + rhs[cidx(G, i, j, k)];
        }
    mg_end(s);
}
// both colours (mg_poisson.F90:32-79); returns this thread's max|resh2|:
// Resmaxg = (max over the CTA or cluster) / h^2 is formed by the caller where
// it is used (the max is exact, so where it is reduced does not change it)
__device__ double mg_relax(MgRun &r, const MgData &d, int m, double *u, const double *rhs) {
    const int n = mgN(d, m), G = n + 2;
    double hh = mgH(d, m), h2 = hh * hh, rm = 0.0;
    const int half = (n * n * n + 1) / 2;
    for (int ipass = 1; ipass <= 2; ipass++) {
        if (d.zbc) mg_boundary_u(r, d, m, u);   // mg_poisson.F90:56 (a wrap on periodic boxes is not needed)
        const MgStep s = mg_begin(r, d, m);
        if (s.on)
            for (int c = s.start; c < half; c += s.stride) {
                int i2, j, k, i;
                if (n == 1) { if (((ipass) & 1) != 0) continue; i = 0; j = 0; k = 0; }
                else {
                    int hn = n / 2;
                    const int lhn = __ffs(hn) - 1;
                    i2 = c & (hn - 1); j = (c >> lhn) & (n - 1); k = c >> (lhn + __ffs(n) - 1);
                    i = 2 * i2 + ((j + k + ipass) & 1);
                }
                const double lap = d.periodic ? mg_lap_sum_wrap(u, G, n, i, j, k) : mg_lap_sum(u, G, i, j, k);
                double resh2 = lap - h2 * rhs[cidx(G, i, j, k)];
                u[cidx(G, i, j, k)] = u[cidx(G, i, j, k)] + (1.0 / 6.0) * resh2;
                double a = fabs(resh2);
                rm = a > rm ? a : rm;
            }
        mg_end(s);
    }
    return rm;
}
__device__ void mg_rstrct(MgRun &r, const MgData &d, int m, double *uc, const double *uf) {   // linear (mg.F90:581-602)
    const int n = mgN(d, m), G = n + 2, Gf = 2 * n + 2, ln = __ffs(n) - 1;
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int c = s.start; c < n * n * n; c += s.stride) {
            int i, j, k;
            mg_ijk(c, n, ln, i, j, k);
            uc[cidx(G, i, j, k)] = rstrct_linear(uf, Gf, 2 * i, 2 * j, 2 * k);
        }
    mg_end(s);
}
// add: uf += the prolongation of uc on uf's interior (the reference's
// mg_interp into a scratch level followed by mg_add: mg_addint, mg.F90:727-731, in one
// step: each sum is the one mg_add forms; uf's ghost layer is left alone,
// which is what adding the scratch level's zero-filled (isolated box) or
// never-read (periodic box) ghost layer does to it)
__device__ void mg_interp(MgRun &r, const MgData &d, int m, double *uf, double *uc, bool cubic,
                          bool add = false) {   // mg.F90:608-633
    const int lc = m + 1, n = mgN(d, m), G = n + 2, nc = mgN(d, lc), Gc = nc + 2, ln = __ffs(n) - 1;
    // Lagrange nodes and weights per fine index, evaluated once per call
    __shared__ int tcw[MG_NMAX][4];
    __shared__ double tww[MG_NMAX][4];
    const bool tri = cubic && nc + 2 >= 4;
    mg_boundary_extrap(r, d, lc, uc);
    mg_boundary_u(r, d, lc, uc);
    {
        const MgStep s = mg_begin(r, d, m);
        if (s.on) {
            if (tri && (int)threadIdx.x < n) cubic_weights((int)threadIdx.x, -1, nc, tcw[threadIdx.x], tww[threadIdx.x]);
            // a small coarse level kept in CTA 0's shared memory, read by every
            // CTA of a large-level step: each CTA copies it first
            const double *src = uc;
            if (s.wide && !mg_wide(r, d, lc) && lc >= r.smem_from) {
                const double *c0 = mg_map_rank(uc, 0);
                for (int t = threadIdx.x; t < Gc * Gc * Gc; t += blockDim.x) r.mirror[t] = c0[t];
                src = r.mirror;
            }
            __syncthreads();
            for (int c = s.start; c < n * n * n; c += s.stride) {
                int i, j, k;
                mg_ijk(c, n, ln, i, j, k);
                const double v = tri ? tricubic_cell_w(src, Gc, tcw[i], tww[i], tcw[j], tww[j], tcw[k], tww[k])
                                     : trilinear_cell(src, Gc, i, j, k, 0, 0, 0);
                const int cf = cidx(G, i, j, k);
                uf[cf] = add ? uf[cf] + v : v;
            }
        }
        mg_end(s);
    }
    if (!add) mg_boundary_fill0(r, d, m, uf);
    mg_boundary_fill0(r, d, lc, uc);
    // the reference wraps uf and uc again here (mg.F90:631-632); uc was
    // wrapped above and is unchanged, and no later step reads the ghost
    // layer of uf before wrapping it (relaxation and residual read periodic
    // images, the next prolongation wraps its coarse level first)
}
// The descent step of mg_lin (mg.F90:185-187) in one step on level v + 1: the
// residual of level v at the eight children of each level-(v+1) cell (the
// expression of mg_resid), their linear restriction (rstrct_linear's sum and
// order) into rhsc, and level v + 1's correction uc zeroed.  The fine
// residual array is not written: nothing reads it before the ascent
// overwrites it.
__device__ void mg_resid_rstrct_fill0(MgRun &r, const MgData &d, int v, double *rhsc, double *u,
                                      const double *rhs, double *uc) {
    const int n = mgN(d, v), G = n + 2, nc = mgN(d, v + 1), Gc = nc + 2, lnc = __ffs(nc) - 1;
    if (d.zbc) mg_boundary_u(r, d, v, u);   // mg_poisson_resid's boundary (mg_poisson.F90:16)
    const double hh = mgH(d, v);
    const double h2i = 1.0 / (hh * hh);
    auto res = [&](int i, int j, int k) {
        const double lap = d.periodic ? mg_lap_sum_wrap(u, G, n, i, j, k) : mg_lap_sum(u, G, i, j, k);
        return -h2i * lap + rhs[cidx(G, i, j, k)];
    };
    const MgStep s = mg_begin(r, d, v + 1);
    if (s.on) {
        for (int c = s.start; c < nc * nc * nc; c += s.stride) {
            int i, j, k;
            mg_ijk(c, nc, lnc, i, j, k);
            const int i0 = 2 * i, j0 = 2 * j, k0 = 2 * k;
            rhsc[cidx(Gc, i, j, k)] = (res(i0, j0, k0) + res(i0 + 1, j0, k0) + res(i0, j0 + 1, k0) +
                                       res(i0, j0, k0 + 1) + res(i0 + 1, j0 + 1, k0) + res(i0 + 1, j0, k0 + 1) +
                                       res(i0, j0 + 1, k0 + 1) + res(i0 + 1, j0 + 1, k0 + 1)) *
                                      (1.0 / 8.0);
        }
        for (int c = s.start; c < Gc * Gc * Gc; c += s.stride) uc[c] = 0.0;
    }
    mg_end(s);
}
__device__ void mg_fill0(MgRun &r, const MgData &d, int m, double *a) {
    const int G = mgN(d, m) + 2;
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int c = s.start; c < G * G * G; c += s.stride) a[c] = 0.0;
    mg_end(s);
}
__device__ void mg_copy(MgRun &r, const MgData &d, int m, double *o, const double *a) {
    const int G = mgN(d, m) + 2;
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int c = s.start; c < G * G * G; c += s.stride) o[c] = a[c];
    mg_end(s);
}
__device__ void mg_addw(MgRun &r, const MgData &d, int m, double *a, const double *da) {
    const int G = mgN(d, m) + 2;
    const MgStep s = mg_begin(r, d, m);
    if (s.on)
        for (int c = s.start; c < G * G * G; c += s.stride) a[c] = a[c] + da[c];
    mg_end(s);
}

// mg_lin (mg.F90:106-218); returns the last Resmaxg (the Resmaxg of every
// earlier mg_relax is overwritten unread, so only the last one is reduced)
__device__ double mg_lin(MgRun &r, const MgData &d, double *sh) {
    double rm = 0.0;   // this thread's max|resh2| of the last mg_relax
    int mr = d.MMax;   // its level
    for (int m = 1; m <= d.MMax; m++) mg_rstrct(r, d, m, d.RHO[m], d.RHO[m - 1]);
    mg_fill0(r, d, d.MMax, d.U[d.MMax]);
    for (int q = 0; q < 2; q++) rm = mg_relax(r, d, d.MMax, d.U[d.MMax], d.RHO[d.MMax]);
    for (int m = d.MMax - 1; m >= 0; m--) {
        mg_interp(r, d, m, d.U[m], d.U[m + 1], true);
        mg_copy(r, d, m, d.RHS[m], d.RHO[m]);
        for (int jc = 1; jc <= 2; jc++) {
            for (int v = m; v <= d.MMax - 1; v++) {
                for (int q = 0; q < 2; q++) rm = mg_relax(r, d, v, d.U[v], d.RHS[v]);
                mr = v;
                mg_resid_rstrct_fill0(r, d, v, d.RHS[v + 1], d.U[v], d.RHS[v], d.U[v + 1]);
            }
            for (int q = 0; q < 2; q++) rm = mg_relax(r, d, d.MMax, d.U[d.MMax], d.RHS[d.MMax]);
            mr = d.MMax;
            for (int v = d.MMax - 1; v >= m; v--) {
                mg_interp(r, d, v, d.U[v], d.U[v + 1], false, true);   // mg_interp + mg_add
                for (int q = 0; q < 2; q++) rm = mg_relax(r, d, v, d.U[v], d.RHS[v]);
                mr = v;
            }
        }
    }
    const double hh = mgH(d, mr);
    // the last relaxation is on level 0 (m = 0 ends the FMG), a large level
    // in cluster mode: every CTA takes part and gets the cluster's maximum
    return mg_max(r, rm, sh, mg_wide(r, d, mr)) / (hh * hh);
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

// cluster special registers (an ordinary launch is a cluster of one CTA)
__device__ __forceinline__ int mg_cluster_rank() {
    int v;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(v));
    return v;
}
__device__ __forceinline__ int mg_cluster_size() {
    int v;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(v));
    return v;
}

// mg_cycle (mg.F90:42-94) with ju = PSI, jrho = SRC, on one CTA or on a
// cluster (launched with a cluster dimension; smem_from must then be above
// every level of at least wide_min cells per edge).  nmax: cap on the
// defect corrections, 10 in the reference.  Dynamic shared memory: the
// U / RES / RHS of levels >= smem_from, then `mirror_doubles` for the copy of
// a small level onto a large one (cluster mode only).
__global__ void __launch_bounds__(512, 1) k_mg_cycle(MgData dg, int smem_from, int *iters_out, int nmax, int wide_min,
                                                     int mirror_doubles) {
    pdl_enter();
    __shared__ double sh[32];
    __shared__ double slot;
    MgData d = dg;
    MgRun r;
    r.rank = mg_cluster_rank();
    r.nct = mg_cluster_size();
    r.wide_min = wide_min;
    r.smem_from = smem_from;
    r.pending = false;
    r.slot = &slot;
    if (r.nct > 1 && d.N < wide_min) {   // no large level: CTA 0 alone, before any cluster barrier
        if (r.rank != 0) return;
        r.nct = 1;
    }
    {
        double *p = mg_dyn_smem();
        for (int m = d.MMax; m >= smem_from; m--) {
            size_t G = (size_t)(d.N >> m) + 2, V = G * G * G;
            d.U[m] = p; p += V;
            d.RES[m] = p; p += V;
            d.RHS[m] = p; p += V;
        }
        r.mirror = p;
        p += mirror_doubles;
        const int64_t tot = p - mg_dyn_smem();
        double *z = mg_dyn_smem();
        for (int64_t t = threadIdx.x; t < tot; t += blockDim.x) z[t] = 0.0;
        __syncthreads();
    }
    if (r.nct > 1) mg_cluster_sync();   // every CTA has started before any reads another's shared memory
    const double errmax = (double)1.e-2f;   // default-real literal (mg.F90:50)
    mg_boundary_fill0(r, d, 0, d.PSI);
    mg_boundary_u(r, d, 0, d.PSI);
    double rhomax = 0.0;
    int it;
    for (it = 1; it <= nmax; it++) {
        mg_resid(r, d, 0, d.RHO[0], d.PSI, d.SRC);
        if (it == 1) {
            const int n = d.N, G = n + 2;
            const MgStep s = mg_begin(r, d, 0);
            double v = 0.0;
            if (s.on)
                for (int c = s.start; c < n * n * n; c += s.stride) {
                    int i, j, k;
                    mg_ijk(c, n, __ffs(n) - 1, i, j, k);
                    double a = fabs(d.RHO[0][cidx(G, i, j, k)]);
                    v = a > v ? a : v;
                }
            rhomax = mg_max(r, v, sh, s.wide);
        }
        double res = mg_lin(r, d, sh);
        mg_addw(r, d, 0, d.PSI, d.U[0]);
        if (res / rhomax < errmax) break;
    }
    if (r.nct > 1) mg_cluster_sync();   // no CTA leaves while another may still read its shared memory
    if (threadIdx.x == 0 && r.rank == 0 && iters_out) *iters_out = it > nmax ? nmax : it;
}

}  // namespace sfm
