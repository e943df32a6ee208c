// sfm_adjoint.cuh -- device side of the adjoint of the converged solve
// (sfm_adjoint; no counterpart in the reference).
//
// The outer loop of the solve stops at the fixed point of its FP64 residual
// on leaf interiors, A x + A_bc phi_bc = SRC, where A is the fmg-level-0
// operator of fmg_poisson_resid (fmg_poisson.F90:217-265): converge_c2p
// (fmg_converge.F90:73-188), the bilinear ghostcell_fix
// (fmg_ghostcell.F90:43-55, 127-199, 312-495), fluxes and fmg_fluxcorrection
// (fmg_poisson.F90:53-124, fmg_reflux.F90:28-258) and the divergence.  The
// functors below apply A^T, the exact transpose of that pipeline, operation
// by operation in reverse order, on FP64 arrays of every block with one
// ghost layer (the fmg-level-0 layout).  Accumulations that several face
// items can make into one cell (coarse cells under the bilinear stencils)
// use FP64 atomics, so the adjoint is reproducible to roundoff, not bitwise.
#pragma once
#include "sfm_kernels_misc.cuh"

namespace sfm {

struct AdjReflux {          // fine face whose neighbour is one level up
    int32_t fine, coarse;
    int8_t dir, lr, oa, ob;
};

__device__ __forceinline__ bool adj_interior(int n, int i, int j, int k) {
    return i >= 0 && i < n && j >= 0 && j < n && k >= 0 && k < n;
}
__device__ __forceinline__ void adj_cell(int64_t r, int G, int &i, int &j, int &k) {
    i = (int)(r % G) - 1;
    j = (int)((r / G) % G) - 1;
    k = (int)(r / ((int64_t)G * G)) - 1;
}

// caller array [nb][(n+2g)^3] -> A [nb][(n+2)^3], interiors only
struct OpAdjIn {
    double *A; const double *in; int n, G, g; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        const int64_t Gi = n + 2 * g;
        A[idx] = adj_interior(n, i, j, k) ? in[b * Gi * Gi * Gi + ((int64_t)(k + g) * Gi + (j + g)) * Gi + (i + g)] : 0.0;
    }
};

// zero everything but leaf interiors
struct OpLeafInterior {
    double *A; const int8_t *skip; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        if (skip[b] || !adj_interior(n, i, j, k)) A[idx] = 0.0;
    }
};

// transpose of converge_c2p_lev: the children of one level push their
// parent octant's adjoint (zeroed) down, 1/8 to each of the 8 fine cells
struct OpConvergeT {
    double *A; const int32_t *parent; const int8_t *oct; int first; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int h = n / 2, per = h * h * h;
        const int b = first + (int)(idx / per);
        const int r = (int)(idx % per);
        const int ic = r % h, jc = (r / h) % h, kc = r / (h * h);
        const int p = parent[b];
        double *pc = A + (int64_t)p * V + cidx(G, ic + oct[3 * b] * h, jc + oct[3 * b + 1] * h, kc + oct[3 * b + 2] * h);
        const double v = *pc * 0.125;
        *pc = 0.0;
        double *cb = A + (int64_t)b * V;
        for (int c = 0; c < 8; c++) cb[cidx(G, 2 * ic + (c & 1), 2 * jc + ((c >> 1) & 1), 2 * kc + (c >> 2))] += v;
    }
};

// transpose of the divergence on leaf blocks: flux adjoints from the
// residual weights g (leaf interiors), written for every cell of every block
struct OpDivT {
    double *fx, *fy, *fz; const double *g; const int8_t *skip; const double *h0; const int32_t *level;
    int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        if (skip[b] || i == n || j == n || k == n) {
            fx[idx] = 0.0; fy[idx] = 0.0; fz[idx] = 0.0;
            return;
        }
        const double hi = 1.0 / hlev(h0, level[b], 0);
        const double *gb = g + b * V;
        auto gv = [&](int a, int c, int d) { return adj_interior(n, a, c, d) ? gb[cidx(G, a, c, d)] : 0.0; };
        const double v = gv(i, j, k);
        fx[idx] = (v - gv(i + 1, j, k)) * hi;
        fy[idx] = (v - gv(i, j + 1, k)) * hi;
        fz[idx] = (v - gv(i, j, k + 1)) * hi;
    }
};

// transpose of fmg_fluxcorrection: the coarse quarter face's adjoint (zeroed)
// goes a quarter to each of the 4 fine face fluxes it averaged
struct OpRefluxT {
    double *fx, *fy, *fz; const AdjReflux *items; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int h = n / 2, per = h * h;
        const AdjReflux it = items[idx / per];
        const int r = (int)(idx % per);
        const int pc = r % h, qc = r / h;
        double *fd = it.dir == 0 ? fx : (it.dir == 1 ? fy : fz);
        const int xc = it.lr == 0 ? n - 1 : -1, xf = it.lr == 0 ? -1 : n - 1;
        int i, j, k;
        put3(it.dir, xc, pc + it.oa * h, qc + it.ob * h, i, j, k);
        double *c = fd + (int64_t)it.coarse * V + cidx(G, i, j, k);
        const double v = *c * 0.25;
        *c = 0.0;
        double *fb = fd + (int64_t)it.fine * V;
        for (int s = 0; s < 4; s++) {
            put3(it.dir, xf, 2 * pc + (s & 1), 2 * qc + (s >> 1), i, j, k);
            fb[cidx(G, i, j, k)] += v;
        }
    }
};

// transpose of the fluxes F_d(i) = (u(i + e_d) - u(i)) / h on leaf blocks,
// i in [-1, n-1]^3: u's adjoint on every cell (zero on covered blocks)
struct OpFluxT {
    double *ub; const double *fx, *fy, *fz; const int8_t *skip; const double *h0; const int32_t *level;
    int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        if (skip[b]) { ub[idx] = 0.0; return; }
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        const double hi = 1.0 / hlev(h0, level[b], 0);
        auto F = [&](const double *f, int a, int c, int d) {
            return (a >= -1 && a < n && c >= -1 && c < n && d >= -1 && d < n) ? f[b * V + cidx(G, a, c, d)] : 0.0;
        };
        double s = F(fx, i - 1, j, k) - F(fx, i, j, k);
        s = s + (F(fy, i, j - 1, k) - F(fy, i, j, k));
        s = s + (F(fz, i, j, k - 1) - F(fz, i, j, k));
        ub[idx] = s * hi;
    }
};

// transpose of one ghost pass (parentlev and samelev of one level and
// direction): each ghost cell's adjoint (zeroed) goes back to what it was
// computed from -- the source plane (same level), or the receiver's two
// inner cells and the coarse layer under the bilinear stencil of
// (10 u0 + 8 uH - 3 uN) / 15 (coarse-fine)
struct OpGhostT {
    double *ub; const FaceItem *items; int n, G; int64_t V; int dir;
    __device__ void operator()(int64_t idx) const {
        const int GT = n + 2;
        const FaceItem it = items[idx / ((int64_t)GT * GT)];
        const int r = (int)(idx % ((int64_t)GT * GT));
        const int p = r % GT - 1, q = r / GT - 1;
        const int xg = it.lr == 0 ? -1 : n;
        int i, j, k;
        put3(dir, xg, p, q, i, j, k);
        double *ud = ub + (int64_t)it.dst * V;
        const double gv = ud[cidx(G, i, j, k)];
        ud[cidx(G, i, j, k)] = 0.0;
        if (gv == 0.0) return;
        double *us = ub + (int64_t)it.src * V;
        if (it.type == 0) {
            const int xs = it.lr == 0 ? n - 1 : 0;
            put3(dir, xs, p, q, i, j, k);
            atomicAdd(us + cidx(G, i, j, k), gv);
            return;
        }
        const int inner = it.lr == 0 ? 1 : -1;
        put3(dir, xg + inner, p, q, i, j, k);
        atomicAdd(ud + cidx(G, i, j, k), (10.0 / 15.0) * gv);
        put3(dir, xg + 2 * inner, p, q, i, j, k);
        atomicAdd(ud + cidx(G, i, j, k), (-3.0 / 15.0) * gv);
        const double hv = (8.0 / 15.0) * gv;
        const int nb2 = n / 2, oa = it.oa * nb2, ob = it.ob * nb2, xc = it.lr == 0 ? n - 1 : 0;
        const int pc = fdiv2(p), qc = fdiv2(q), p1 = near_(p, pc), q1 = near_(q, qc);
        put3(dir, xc, pc + oa, qc + ob, i, j, k);
        atomicAdd(us + cidx(G, i, j, k), (9.0 / 16.0) * hv);
        put3(dir, xc, p1 + oa, q1 + ob, i, j, k);
        atomicAdd(us + cidx(G, i, j, k), (1.0 / 16.0) * hv);
        put3(dir, xc, pc + oa, q1 + ob, i, j, k);
        atomicAdd(us + cidx(G, i, j, k), (3.0 / 16.0) * hv);
        put3(dir, xc, p1 + oa, qc + ob, i, j, k);
        atomicAdd(us + cidx(G, i, j, k), (3.0 / 16.0) * hv);
    }
};

// preconditioner hand-off: R = v / dv on leaf interiors, else 0 ...
template <class T>
struct OpPrecIn {
    T *R; const double *v; const int8_t *skip; const double *h0; const int32_t *level; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        const double h = hlev(h0, level[b], 0);
        R[idx] = (!skip[b] && adj_interior(n, i, j, k)) ? (T)(v[idx] / (h * h * h)) : (T)0;
    }
};
// ... and z = u * dv back
template <class T>
struct OpPrecOut {
    double *z; const T *U; const int8_t *skip; const double *h0; const int32_t *level; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        const double h = hlev(h0, level[b], 0);
        z[idx] = (!skip[b] && adj_interior(n, i, j, k)) ? (double)U[idx] * (h * h * h) : 0.0;
    }
};

// y = y + a x
struct OpAxpy {
    double *y; const double *x; double a;
    __device__ void operator()(int64_t idx) const { y[idx] = y[idx] + a * x[idx]; }
};
struct OpAxpyLeafConst {   // A += c on leaf interiors
    double *A; double c; const int8_t *skip; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        if (!skip[b] && adj_interior(n, i, j, k)) A[idx] = A[idx] + c;
    }
};
struct OpScale {
    double *y; double a;
    __device__ void operator()(int64_t idx) const { y[idx] = y[idx] * a; }
};
struct OpSubArr {   // o = a - b
    double *o; const double *a, *b;
    __device__ void operator()(int64_t idx) const { o[idx] = a[idx] - b[idx]; }
};

// per-leaf-block partial sums of a*b (of a when b is null) over the
// interior, in cell order
struct OpBlockDot {
    const double *a, *b; const int32_t *blocks; double *psum; int n, G; int64_t V;
    __device__ void operator()(int64_t q) const {
        const int64_t off = (int64_t)blocks[q] * V;
        double s = 0.0;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    const int64_t c = off + cidx(G, i, j, k);
                    s = s + (b ? a[c] * b[c] : a[c]);
                }
        psum[q] = s;
    }
};
// ordered sum of cnt partials into *out: one warp, contiguous chunks per lane
__global__ void __launch_bounds__(32) k_sum_ordered(const double *psum, int cnt, double *out) {
    pdl_enter();
    __shared__ double part[32];
    const int lane = threadIdx.x;
    const int chunk = (cnt + 31) / 32;
    double s = 0.0;
    for (int q = lane * chunk; q < cnt && q < (lane + 1) * chunk; q++) s = s + psum[q];
    part[lane] = s;
    __syncwarp();
    if (lane == 0) {
        double t = 0.0;
        for (int l = 0; l < 32; l++) t = t + part[l];
        *out = t;
    }
}

// moment kernels T_q(x) of the isolated boundary (the factors of rho dv in
// the moment sums, fmg_boundary_phys_sphere.F90:160-186, and the l = 4
// extension), and the normalisations nrm_q with mom_q = -nrm_q sum T_q rho dv
__device__ inline void adj_moment_terms(double x, double y, double z, double t[25]) {
    const double r2 = x * x + y * y + z * z, r = sqrt(r2), r3 = r2 * r, rc = sqrt(x * x + y * y);
    const double cost = z / r, sint = rc / r, cosp = x / rc, sinp = y / rc;
    const double c2 = cost * cost, s2 = sint * sint, cp2 = cosp * cosp, sp2 = sinp * sinp;
    t[0] = 1.0; t[1] = r * cost; t[2] = r * sint * cosp; t[3] = r * sint * sinp;
    t[4] = r2 * (3 * c2 - 1); t[5] = r2 * sint * cost * cosp; t[6] = r2 * sint * cost * sinp;
    t[7] = r2 * s2 * (cp2 - sp2); t[8] = r2 * s2 * 2 * sinp * cosp;
    t[9] = r3 * cost * (5 * c2 - 3); t[10] = r3 * sint * (5 * c2 - 1) * cosp; t[11] = r3 * sint * (5 * c2 - 1) * sinp;
    t[12] = r3 * cost * s2 * (cp2 - sp2); t[13] = r3 * cost * s2 * 2 * sinp * cosp;
    t[14] = r3 * s2 * sint * cosp * (cp2 - 3 * sp2); t[15] = r3 * s2 * sint * sinp * (3 * cp2 - sp2);
    const double r4 = r2 * r2, cos2p = cp2 - sp2, sin2p = 2 * sinp * cosp;
    const double cos3p = cosp * (cp2 - 3 * sp2), sin3p = sinp * (3 * cp2 - sp2);
    const double cos4p = cos2p * cos2p - sin2p * sin2p, sin4p = 2 * sin2p * cos2p;
    t[16] = r4 * (35 * c2 * c2 - 30 * c2 + 3); t[17] = r4 * sint * cost * (7 * c2 - 3) * cosp;
    t[18] = r4 * sint * cost * (7 * c2 - 3) * sinp; t[19] = r4 * s2 * (7 * c2 - 1) * cos2p;
    t[20] = r4 * s2 * (7 * c2 - 1) * sin2p; t[21] = r4 * s2 * sint * cost * cos3p;
    t[22] = r4 * s2 * sint * cost * sin3p; t[23] = r4 * s2 * s2 * cos4p; t[24] = r4 * s2 * s2 * sin4p;
}
__device__ inline double adj_moment_norm(int q) {
    const double pi = 3.14159265358979323846;
    switch (q) {
        case 0: case 1: return 1 / (4 * pi);
        case 2: case 3: return 1 / (8 * pi);
        case 4: return 1 / (16 * pi);
        case 5: case 6: return 3 / (8 * pi);
        case 7: case 8: return 3 / (32 * pi);
        case 9: return 1 / (16 * pi);
        case 10: case 11: return 3 / (64 * pi);
        case 12: case 13: return 15 / (32 * pi);
        case 14: case 15: return 5 / (64 * pi);
        case 16: return 1 / (4 * pi * 64);
        case 17: case 18: return 5 / (4 * pi * 8);
        case 19: case 20: return 5 / (4 * pi * 16);
        case 21: case 22: return 35 / (4 * pi * 8);
        default: return 35 / (4 * pi * 64);
    }
}

// beta_q partial per boundary face: sum over the face's ghost cells c of
// E_q(x_c) * (-ub_c), E_q the potential of a unit moment q; a cell shared
// with a touching face of a lower direction is counted there only
struct OpBcBeta {
    const double *ub; const BFace *faces; const int8_t *touch; const double *x0; const double *h0;
    const int32_t *level; double *part; int n, G; int64_t V; int lmax;
    __device__ void operator()(int64_t fi) const {
        const BFace f = faces[fi];
        const int dir = f.face >> 1, lr = f.face & 1, b = f.b;
        const double h = h0[level[b]];
        const double *xb = x0 + 3 * b;
        const int xg = lr == 0 ? -1 : n;
        const int kmax = lmax >= 4 ? 25 : 16;
        double acc[25];
        for (int q = 0; q < 25; q++) acc[q] = 0.0;
        for (int qq = -1; qq <= n; qq++)
            for (int pp = -1; pp <= n; pp++) {
                int c[3];
                put3(dir, xg, pp, qq, c[0], c[1], c[2]);
                bool dup = false;
                for (int d = 0; d < dir; d++) {
                    if (c[d] == -1 && touch[6 * b + 2 * d]) dup = true;
                    if (c[d] == n && touch[6 * b + 1 + 2 * d]) dup = true;
                }
                if (dup) continue;
                const double w = -ub[(int64_t)b * V + cidx(G, c[0], c[1], c[2])];
                if (w == 0.0) continue;
                const double x = xb[0] + (double)c[0] * h, y = xb[1] + (double)c[1] * h, z = xb[2] + (double)c[2] * h;
                for (int q = 0; q < kmax; q++) {
                    double e[25];
                    for (int s = 0; s < 25; s++) e[s] = 0.0;
                    e[q] = 1.0;
                    acc[q] = acc[q] + w * multipole_eval(e, lmax, x, y, z);
                }
            }
        for (int q = 0; q < 25; q++) part[fi * 25 + q] = acc[q];
    }
};
// beta_q = ordered sum of the face partials (one thread per q)
__global__ void k_bc_beta_combine(const double *part, int nfaces, double *beta) {
    pdl_enter();
    const int q = threadIdx.x;
    if (q >= 25) return;
    double s = 0.0;
    for (int f = 0; f < nfaces; f++) s = s + part[(int64_t)f * 25 + q];
    beta[q] = s;
}
// dJ/dSRC on base-level interiors through the moments (masked cells get 0)
struct OpMomentT {
    double *S; const double *beta; const double *x0; const double *h0; int first; int n, G; int64_t V;
    double rad2; int lmax;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        const int b = first + (int)(idx / per);
        const int r = (int)(idx % per);
        const int i = r % n, j = (r / n) % n, k = r / (n * n);
        const double h = h0[0];
        const double x = x0[3 * b] + (double)i * h, y = x0[3 * b + 1] + (double)j * h, z = x0[3 * b + 2] + (double)k * h;
        double v = 0.0;
        if (x * x + y * y + z * z < rad2) {
            double t[25];
            adj_moment_terms(x, y, z, t);
            const int kmax = lmax >= 4 ? 25 : 16;
            for (int q = 0; q < kmax; q++) v += beta[q] * (-adj_moment_norm(q)) * t[q] * (h * h * h);
        }
        S[(int64_t)b * V + cidx(G, i, j, k)] = v;
    }
};
// S += mask * lambda on leaf interiors, S = 0 elsewhere (mask: inside the
// sphere radius, or everywhere when rad2 < 0)
struct OpAddMaskedLambda {
    double *S; const double *lam; const int8_t *skip; const double *x0; const double *h0; const int32_t *level;
    int n, G; int64_t V; double rad2;
    __device__ void operator()(int64_t idx) const {
        const int64_t b = idx / V;
        int i, j, k;
        adj_cell(idx % V, G, i, j, k);
        if (skip[b] || !adj_interior(n, i, j, k)) { S[idx] = 0.0; return; }
        bool in = true;
        if (rad2 >= 0.0) {
            const double h = h0[level[b]];
            const double x = x0[3 * b] + (double)i * h, y = x0[3 * b + 1] + (double)j * h, z = x0[3 * b + 2] + (double)k * h;
            in = x * x + y * y + z * z < rad2;
        }
        S[idx] = S[idx] + (in ? lam[idx] : 0.0);
    }
};
// dJ/drho = four_pi_G (S - dv * corr) on leaf interiors of the caller layout
struct OpAdjOut {
    double *out; const double *S; const int8_t *skip; const double *h0; const int32_t *level;
    int n, G, g; int64_t V; double fourpiG, corr;
    __device__ void operator()(int64_t idx) const {
        const int64_t Gi = n + 2 * g;
        const int64_t Vi = Gi * Gi * Gi;
        const int64_t b = idx / Vi;
        const int64_t r = idx % Vi;
        const int i = (int)(r % Gi) - g, j = (int)((r / Gi) % Gi) - g, k = (int)(r / (Gi * Gi)) - g;
        if (skip[b] || !adj_interior(n, i, j, k)) { out[idx] = 0.0; return; }
        const double h = hlev(h0, level[b], 0);
        out[idx] = fourpiG * (S[b * V + cidx(G, i, j, k)] - (h * h * h) * corr);
    }
};

}  // namespace sfm
