// sfm_kernels_misc.cuh -- set-up, boundary, reduction and base-grid kernels.
#pragma once
#include "sfm_device.cuh"

namespace sfm {

// ---------------------------------------------------------------------------
// fmg_make_physvar / fmg_prepare_interp (fmg_data_if.F90:13-84,176-217):
// U := psi (warm start), RHO := rho * 4 pi G on (-1:n)^3, from the caller's
// arrays with `g` ghost layers.  Non-finite inputs raise *bad.
// ---------------------------------------------------------------------------
template <class TR>
struct OpPhysvar {
    double *U; TR *R; const double *rho; const double *psi; int n, G, g; int64_t V; double fourpiG; int *bad;
    __device__ void operator()(int64_t idx) const {
        int64_t b = idx / V;
        int r = (int)(idx % V);
        int i = r % G - 1, j = (r / G) % G - 1, k = r / (G * G) - 1;
        const int Gi = n + 2 * g;
        int64_t s = b * (int64_t)Gi * Gi * Gi + ((int64_t)(k + g) * Gi + (j + g)) * Gi + (i + g);
        double rv = rho[s], pv = psi ? psi[s] : 0.0;
        if (!isfinite(rv) || !isfinite(pv)) *bad = 1;
        U[idx] = pv;
        R[idx] = (TR)(rv * fourpiG);
    }
};

// per-block interior sum, sequential in (i fastest) order as Fortran SUM
template <class T>
struct OpBlockSum {
    const T *a; const int32_t *blocks; double *out; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const T *ab = a + (int64_t)blocks[idx] * V;
        double s = 0.0;
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) s = s + (double)ab[cidx(G, i, j, k)];
        out[idx] = s;
    }
};

// leaf-volume mean of RHO (fmg_data_if.F90:59-77): mass and volume summed
// block after block in level order, then rho_ave -> *out
__global__ void k_mean_combine(const double *psum, const int32_t *blocks, int nblk, const int32_t *level,
                               const double *h0, int n, double *out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double mass = 0.0, vol = 0.0;
    for (int q = 0; q < nblk; q++) {
        double hd = h0[level[blocks[q]]];
        double dv = hd * hd * hd;
        mass = mass + psum[q] * dv;
        vol = vol + (double)(n * n * n) * dv;
    }
    *out = mass / vol;
}

// vmg_zeroAverage (vmg.F90:900-916) via fmg_ave (fmg_data.F90:730-769)
__global__ void k_ave_combine(const double *psum, int nblk, int n, double *out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double ave = 0.0;
    for (int q = 0; q < nblk; q++) ave = ave + psum[q];
    *out = nblk == 0 ? 0.0 : ave / (double)(n * n * n * nblk);
}

template <class T>
struct OpSubScalarAll {      // a := a - *s over whole arrays
    T *a; const double *s;
    __device__ void operator()(int64_t idx) const { a[idx] = a[idx] - (T)(*s); }
};
template <class T>
struct OpSubScalarInterior { // a := a - *s on the interior of consecutive blocks
    T *a; const double *s; int first, n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = first + (int)(idx / per);
        int r = (int)(idx % per);
        int64_t c = (int64_t)b * V + cidx(G, r % n, (r / n) % n, r / (n * n));
        a[c] = a[c] - (T)(*s);
    }
};

// ---------------------------------------------------------------------------
// isolated boundary (fmg_boundary_phys_sphere.F90:81-354)
// ---------------------------------------------------------------------------
// z-mirror plane: u(:,:,-1) = u(:,:,0) over the whole transverse range of
// the listed blocks (those touching the box's z-min face;
// fmg_boundary_phys_zmirror.F90:66-80): the first G^2 values of a block get
// the next G^2
template <class T>
struct OpMirrorZ {
    T *u; const int32_t *blocks; int G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int64_t per = (int64_t)G * G;
        const int64_t b = blocks[idx / per], t = idx % per;
        u[b * V + t] = u[b * V + t + per];
    }
};
// the z-periodic cylinders' masks and ghosts
// (fmg_boundary_phys_cyl_zperiodic.F90:120-232, ..._mask_zperiodic.F90:129)
struct OpCylMask {           // rho := 0 where x^2+y^2 >= rad2, all cells of all blocks
    double *R; const double *x0; const double *h0; const int32_t *level; int n, G; int64_t V; double rad2;
    __device__ void operator()(int64_t idx) const {
        int64_t b = idx / V;
        int r = (int)(idx % V);
        int i = r % G - 1, j = (r / G) % G - 1;
        double h = h0[level[b]];
        double x = x0[3 * b] + (double)i * h, y = x0[3 * b + 1] + (double)j * h;
        if (x * x + y * y >= rad2) R[idx] = 0.0;
    }
};
struct OpRhoMask {           // rho := 0 where rho < MP_rhomask, all cells of all blocks
    double *R; double thresh;
    __device__ void operator()(int64_t idx) const {
        if (R[idx] < thresh) R[idx] = 0.0;
    }
};
struct OpCylGhost {          // a00 ln(r) on the first ghost layer of the x and y boundary faces
    double *U; const BFace *faces; const double *lnr; const double *mom; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int GT = n + 2;
        int64_t it = idx / (GT * GT);
        int r = (int)(idx - it * GT * GT);
        BFace bf = faces[it];
        int dir = bf.face >> 1, lr = bf.face & 1, i, j, k;
        if (dir == 2) return;   // z is periodic
        put3(dir, lr == 0 ? -1 : n, r % GT - 1, r / GT - 1, i, j, k);
        U[(int64_t)bf.b * V + cidx(G, i, j, k)] = lnr[idx] * mom[0];
    }
};
struct OpSphereMask {        // rho := 0 where x^2+y^2+z^2 >= rad2, all cells of all blocks
    double *R; const double *x0; const double *h0; const int32_t *level; int n, G; int64_t V; double rad2;
    __device__ void operator()(int64_t idx) const {
        int64_t b = idx / V;
        int r = (int)(idx % V);
        int i = r % G - 1, j = (r / G) % G - 1, k = r / (G * G) - 1;
        double h = h0[level[b]];
        double x = x0[3 * b] + (double)i * h, y = x0[3 * b + 1] + (double)j * h, z = x0[3 * b + 2] + (double)k * h;
        if (x * x + y * y + z * z >= rad2) R[idx] = 0.0;
    }
};

// Multipole moments a_lm of the masked source over the base-level interior
// cells (fmg_boundary_phys_sphere.F90:132-242; the l = 4 terms extend the
// reference).  The reference accumulates every moment in one running sum
// over the base blocks in list order and, inside a block, k, j, i; the two
// kernels below keep that order, so the moments -- and with them the whole
// isolated-boundary solve -- are bit-identical to a serial evaluation:
// k_moment_terms evaluates each cell's 25 terms in parallel (the reference's
// expressions, left to right), k_moments_ordered adds them in cell order,
// one lane per moment, with the loads running ahead of the dependent adds.
constexpr int kMomentTerms = 25;
__global__ void k_moment_terms(const double *R, const double *x0, const double *h0, int n, int G, int64_t V,
                               int nbase, int lmax, double *T /* [nbase n^3][25] */) {
    pdl_enter();
    const int64_t ncell = (int64_t)nbase * n * n * n;
    const double h = h0[0], dv = h * h * h;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
        const int per = n * n * n;
        const int b = (int)(c / per), r = (int)(c - (int64_t)b * per);
        const int i = r % n, j = (r / n) % n, k = r / (n * n);
        double x = x0[3 * b] + (double)i * h, y = x0[3 * b + 1] + (double)j * h, z = x0[3 * b + 2] + (double)k * h;
        double r2 = x * x + y * y + z * z;
        double rr = sqrt(r2);
        double r3 = r2 * rr;
        double rc = sqrt(x * x + y * y);
        double ri = 1 / rr, rci = 1 / rc;
        double cost = z * ri, sint = rc * ri, cosp = x * rci, sinp = y * rci;
        double rhodv = R[(int64_t)b * V + cidx(G, i, j, k)] * dv;
        double *t = T + c * kMomentTerms;
        t[0] = rhodv;
        t[1] = rhodv * rr * cost;
        t[2] = rhodv * rr * sint * cosp;
        t[3] = rhodv * rr * sint * sinp;
        t[4] = rhodv * r2 * (3 * (cost * cost) - 1);
        t[5] = rhodv * r2 * sint * cost * cosp;
        t[6] = rhodv * r2 * sint * cost * sinp;
        t[7] = rhodv * r2 * (sint * sint) * ((cosp * cosp) - (sinp * sinp));
        t[8] = rhodv * r2 * (sint * sint) * 2 * sinp * cosp;
        t[9] = rhodv * r3 * cost * (5 * (cost * cost) - 3);
        t[10] = rhodv * r3 * sint * (5 * (cost * cost) - 1) * cosp;
        t[11] = rhodv * r3 * sint * (5 * (cost * cost) - 1) * sinp;
        t[12] = rhodv * r3 * cost * (sint * sint) * ((cosp * cosp) - (sinp * sinp));
        t[13] = rhodv * r3 * cost * (sint * sint) * 2 * sinp * cosp;
        t[14] = rhodv * r3 * (sint * sint * sint) * cosp * ((cosp * cosp) - 3 * (sinp * sinp));
        t[15] = rhodv * r3 * (sint * sint * sint) * sinp * (3 * (cosp * cosp) - (sinp * sinp));
        if (lmax >= 4) {
            double r4 = r2 * r2, c2 = cost * cost, s2 = sint * sint;
            double cos2p = (cosp * cosp) - (sinp * sinp), sin2p = 2 * sinp * cosp;
            double cos3p = cosp * ((cosp * cosp) - 3 * (sinp * sinp));
            double sin3p = sinp * (3 * (cosp * cosp) - (sinp * sinp));
            double cos4p = cos2p * cos2p - sin2p * sin2p, sin4p = 2 * sin2p * cos2p;
            t[16] = rhodv * r4 * (35 * (c2 * c2) - 30 * c2 + 3);
            t[17] = rhodv * r4 * sint * cost * (7 * c2 - 3) * cosp;
            t[18] = rhodv * r4 * sint * cost * (7 * c2 - 3) * sinp;
            t[19] = rhodv * r4 * s2 * (7 * c2 - 1) * cos2p;
            t[20] = rhodv * r4 * s2 * (7 * c2 - 1) * sin2p;
            t[21] = rhodv * r4 * s2 * sint * cost * cos3p;
            t[22] = rhodv * r4 * s2 * sint * cost * sin3p;
            t[23] = rhodv * r4 * (s2 * s2) * cos4p;
            t[24] = rhodv * r4 * (s2 * s2) * sin4p;
        } else {
            for (int m = 16; m < kMomentTerms; m++) t[m] = 0.0;
        }
    }
}

// normalisations (fmg_boundary_phys_sphere.F90:227-242; l = 4 extension)
__device__ __forceinline__ double moment_norm(int m, double a) {
    const double pi = 3.141592653589793;
    switch (m) {
        case 0: return -a / (4.0 * pi);
        case 1: return -a / (4.0 * pi);
        case 2: return -a / (8.0 * pi);
        case 3: return -a / (8.0 * pi);
        case 4: return -a / (16.0 * pi);
        case 5: return -a / (8.0 * pi) * 3.0;
        case 6: return -a / (8.0 * pi) * 3.0;
        case 7: return -a / (32.0 * pi) * 3.0;
        case 8: return -a / (32.0 * pi) * 3.0;
        case 9: return -a / (16.0 * pi);
        case 10: return -a / (64.0 * pi) * 3.0;
        case 11: return -a / (64.0 * pi) * 3.0;
        case 12: return -a / (32.0 * pi) * 15.0;
        case 13: return -a / (32.0 * pi) * 15.0;
        case 14: return -a / (64.0 * pi) * 5.0;
        case 15: return -a / (64.0 * pi) * 5.0;
        case 16: return -a / (4.0 * pi) * (1.0 / 64.0);
        case 17: return -a / (4.0 * pi) * (5.0 / 8.0);
        case 18: return -a / (4.0 * pi) * (5.0 / 8.0);
        case 19: return -a / (4.0 * pi) * (5.0 / 16.0);
        case 20: return -a / (4.0 * pi) * (5.0 / 16.0);
        case 21: return -a / (4.0 * pi) * (35.0 / 8.0);
        case 22: return -a / (4.0 * pi) * (35.0 / 8.0);
        case 23: return -a / (4.0 * pi) * (35.0 / 64.0);
        default: return -a / (4.0 * pi) * (35.0 / 64.0);
    }
}

// factor of moment term m on a z-mirror box: the mirror image doubles the
// terms even in z (l + m even) and cancels the odd ones
// (fmg_boundary_phys_zmirror.F90:243-258; l = 4 by the same rule)
__device__ __forceinline__ double zmirror_factor(int m) {
    // (l + m) parity of the terms a00, a10, a11r, a11i, a20, ..., a33i, l = 4
    constexpr unsigned kOdd = (1u << 1) | (1u << 5) | (1u << 6) | (1u << 9) | (1u << 12) | (1u << 13) | (1u << 17) |
                              (1u << 18) | (1u << 21) | (1u << 22);
    return ((kOdd >> m) & 1u) ? 0.0 : 2.0;
}
// one warp; lane m < 25 sums term m over the cells in order
// mode 0: the sphere's normalisations; 1: the same times the z-mirror
// factors; 2: the z-periodic cylinders' a00 = (sum of term 0) / zlen / pi2
// (cyl_zperiodic.F90:197) in mom[0]
__global__ void __launch_bounds__(32) k_moments_ordered(const double *__restrict__ T, int64_t ncell, double *mom,
                                                         int mode, double zlen, double pi2) {
    pdl_enter();
    const int m = threadIdx.x;
    if (m >= kMomentTerms) return;
    constexpr int U = 16;   // loads issued ahead of the dependent adds
    double a = 0.0;
    int64_t c = 0;
    for (; c + U <= ncell; c += U) {
        double t[U];
#pragma unroll
        for (int u = 0; u < U; u++) t[u] = T[(c + u) * kMomentTerms + m];
#pragma unroll
        for (int u = 0; u < U; u++) a = a + t[u];
    }
    for (; c < ncell; c++) a = a + T[c * kMomentTerms + m];
    if (mode == 2) {
        if (m == 0) mom[0] = a / zlen / pi2;
        return;
    }
    mom[m] = mode == 1 ? moment_norm(m, a) * zmirror_factor(m) : moment_norm(m, a);
}

// U00..U33 (sphere.F90:267-293) and the l = 4 terms
__device__ __forceinline__ double multipole_eval(const double *m, int lmax, double x, double y, double z) {
    double r2i = 1 / (x * x + y * y + z * z);
    double ri = sqrt(r2i);
    double r3i = r2i * ri;
    double r4i = r2i * r2i;
    double rc = sqrt(x * x + y * y);
    double rci = 1 / rc;
    double cost = z * ri, sint = rc * ri, cosp = x * rci, sinp = y * rci;
    double U00 = ri * m[0];
    double U10 = r2i * cost * m[1];
    double U11 = r2i * sint * (cosp * m[2] + sinp * m[3]) * 2;
    double U20 = r3i * (3 * (cost * cost) - 1) * m[4];
    double U21 = r3i * sint * cost * (cosp * m[5] + sinp * m[6]) * 2;
    double U22 = r3i * (sint * sint) * (((cosp * cosp) - (sinp * sinp)) * m[7] + 2 * sinp * cosp * m[8]) * 2;
    double U30 = r4i * cost * (5 * (cost * cost) - 3) * m[9];
    double U31 = r4i * sint * (5 * (cost * cost) - 1) * (cosp * m[10] + sinp * m[11]) * 2;
    double U32 = r4i * cost * (sint * sint) * (((cosp * cosp) - (sinp * sinp)) * m[12] + 2 * sinp * cosp * m[13]) * 2;
    double U33 = r4i * (sint * sint * sint) * (cosp * ((cosp * cosp) - 3 * (sinp * sinp)) * m[14]
                                              + sinp * (3 * (cosp * cosp) - (sinp * sinp)) * m[15]) * 2;
    double ub = U00 + U10 + U11 + U20 + U21 + U22 + U30 + U31 + U32 + U33;
    if (lmax >= 4) {
        double r5i = r4i * ri, c2 = cost * cost, s2 = sint * sint;
        double cos2p = (cosp * cosp) - (sinp * sinp), sin2p = 2 * sinp * cosp;
        double cos3p = cosp * ((cosp * cosp) - 3 * (sinp * sinp));
        double sin3p = sinp * (3 * (cosp * cosp) - (sinp * sinp));
        double cos4p = cos2p * cos2p - sin2p * sin2p, sin4p = 2 * sin2p * cos2p;
        double U40 = r5i * (35 * (c2 * c2) - 30 * c2 + 3) * m[16];
        double U41 = r5i * sint * cost * (7 * c2 - 3) * (cosp * m[17] + sinp * m[18]);
        double U42 = r5i * s2 * (7 * c2 - 1) * (cos2p * m[19] + sin2p * m[20]);
        double U43 = r5i * s2 * sint * cost * (cos3p * m[21] + sin3p * m[22]);
        double U44 = r5i * (s2 * s2) * (cos4p * m[23] + sin4p * m[24]);
        ub = ub + U40 + U41 + U42 + U43 + U44;
    }
    return ub;
}

struct OpSphereGhost {       // potential on the first ghost layer of boundary faces
    double *U; const BFace *faces; const double *mom; const double *x0; const double *h0; const int32_t *level;
    int n, G; int64_t V; int lmax;
    __device__ void operator()(int64_t idx) const {
        const int GT = n + 2;
        int64_t it = idx / (GT * GT);
        int r = (int)(idx - it * GT * GT);
        BFace bf = faces[it];
        int dir = bf.face >> 1, lr = bf.face & 1, i, j, k;
        put3(dir, lr == 0 ? -1 : n, r % GT - 1, r / GT - 1, i, j, k);
        double h = h0[level[bf.b]];
        const double *xb = x0 + 3 * (int64_t)bf.b;
        U[(int64_t)bf.b * V + cidx(G, i, j, k)] =
            multipole_eval(mom, lmax, xb[0] + (double)i * h, xb[1] + (double)j * h, xb[2] + (double)k * h);
    }
};

// ---------------------------------------------------------------------------
// fmg_psi2g (fmg_poisson.F90:4-49) into the caller's layout, and
// fmg_restore_u (fmg_data_if.F90:275-294)
// ---------------------------------------------------------------------------
struct OpPsi2g {
    double *g; const double *U; const int8_t *skip; const int32_t *level; const double *h0;
    const int32_t *rslot; const double *rbuf; int n, G, gw; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = (int)(idx / per);
        int r = (int)(idx % per);
        int i = r % n, j = (r / n) % n, k = r / (n * n);
        const int Gi = n + 2 * gw;
        const int64_t Vi = (int64_t)Gi * Gi * Gi;
        int64_t s = ((int64_t)(k + gw) * Gi + (j + gw)) * Gi + (i + gw);
        double *gx = g + (int64_t)b * 3 * Vi, *gy = gx + Vi, *gz = gy + Vi;
        double hi = 1.0 / hlev(h0, level[b], 0);
        const double *ub = U + (int64_t)b * V;
        if (skip[b]) {
            gx[s] = -((ub[cidx(G, i + 1, j, k)] - ub[cidx(G, i - 1, j, k)]) * hi * 0.5);
            gy[s] = -((ub[cidx(G, i, j + 1, k)] - ub[cidx(G, i, j - 1, k)]) * hi * 0.5);
            gz[s] = -((ub[cidx(G, i, j, k + 1)] - ub[cidx(G, i, j, k - 1)]) * hi * 0.5);
        } else {
            Flux<double> F{ub, G, n, hi, rslot, rbuf, b};
            gx[s] = -((F(0, i, j, k) + F(0, i - 1, j, k)) * 0.5);
            gy[s] = -((F(1, i, j, k) + F(1, i, j - 1, k)) * 0.5);
            gz[s] = -((F(2, i, j, k) + F(2, i, j, k - 1)) * 0.5);
        }
    }
};
struct OpRestore {
    double *psi; const double *U; int n, G, gw; int64_t V;
    __device__ void operator()(int64_t idx) const {
        int64_t b = idx / V;
        int r = (int)(idx % V);
        int i = r % G - 1, j = (r / G) % G - 1, k = r / (G * G) - 1;
        const int Gi = n + 2 * gw;
        psi[b * (int64_t)Gi * Gi * Gi + ((int64_t)(k + gw) * Gi + (j + gw)) * Gi + (i + gw)] = U[idx];
    }
};

// ---------------------------------------------------------------------------
// vmg_tau_crop (vmg.F90:463-505): zero the parent's boundary plane behind
// every face of a child whose neighbour is one level up
// ---------------------------------------------------------------------------
template <class T>
struct OpTauCrop {
    T *tau; const BFace *faces; const int32_t *parent; int n, G; int64_t V;
    __device__ void operator()(int64_t idx) const {
        const int GT = n + 2;
        int64_t it = idx / (GT * GT);
        int r = (int)(idx - it * GT * GT);
        BFace bf = faces[it];
        int dir = bf.face >> 1, lr = bf.face & 1, i, j, k;
        put3(dir, lr == 0 ? 0 : n - 1, r % GT - 1, r / GT - 1, i, j, k);
        tau[(int64_t)parent[bf.b] * V + cidx(G, i, j, k)] = (T)0;
    }
};

// tau on fine blocks: 0 everywhere, -(div F)/h inside (vmg_poisson.F90:18-35)
template <class T>
struct OpTauFine {
    T *tau; const T *u; int first, n, G; int64_t V; T hi;
    __device__ void operator()(int64_t idx) const {
        int b = first + (int)(idx / V);
        int r = (int)(idx % V);
        int i = r % G - 1, j = (r / G) % G - 1, k = r / (G * G) - 1;
        T v = (T)0;
        if (i >= 0 && i < n && j >= 0 && j < n && k >= 0 && k < n) {
            Flux<T> F{u + (int64_t)b * V, G, n, hi, nullptr, nullptr, b};
            v = -(F.div(i, j, k) * hi);
        }
        tau[(int64_t)b * V + r] = v;
    }
};
// tau += (div F)/h on parents with children (vmg_poisson.F90:40-57)
template <class T>
struct OpTauParent {
    T *tau; const T *u; const int32_t *blocks; int n, G; int64_t V; T hi;
    __device__ void operator()(int64_t idx) const {
        const int per = n * n * n;
        int b = blocks[idx / per];
        int r = (int)(idx % per);
        int i = r % n, j = (r / n) % n, k = r / (n * n);
        Flux<T> F{u + (int64_t)b * V, G, n, hi, nullptr, nullptr, b};
        int64_t c = (int64_t)b * V + cidx(G, i, j, k);
        tau[c] = tau[c] + F.div(i, j, k) * hi;
    }
};

// ---------------------------------------------------------------------------
// base grid <-> base blocks (mg_dataPrepare / mg_dataRestore,
// mg_data.F90:179-330)
// ---------------------------------------------------------------------------
template <class T>
struct OpMgGather {
    double *S, *P; const T *rhs, *u; const int32_t *baseIdx; int ngb0, ngb1, n, G, N; int64_t V;
    __device__ void operator()(int64_t idx) const {
        int N3 = N;   // cells per base-grid edge
        int I = (int)(idx % N3), J = (int)((idx / N3) % N3), K = (int)(idx / ((int64_t)N3 * N3));
        int ib = I / n, jb = J / n, kb = K / n;
        int b = baseIdx[((int64_t)kb * ngb1 + jb) * ngb0 + ib];
        int64_t c = (int64_t)b * V + cidx(G, I - ib * n, J - jb * n, K - kb * n);
        int64_t m = cidx(N + 2, I, J, K);
        S[m] = (double)rhs[c];
        P[m] = (double)u[c];
    }
};
template <class T>
struct OpMgScatter {
    T *u; const double *P; const int32_t *baseIdx; int ngb0, ngb1, n, G, N; int64_t V;
    __device__ void operator()(int64_t idx) const {
        int I = (int)(idx % N), J = (int)((idx / N) % N), K = (int)(idx / ((int64_t)N * N));
        int ib = I / n, jb = J / n, kb = K / n;
        int b = baseIdx[((int64_t)kb * ngb1 + jb) * ngb0 + ib];
        u[(int64_t)b * V + cidx(G, I - ib * n, J - jb * n, K - kb * n)] = (T)P[cidx(N + 2, I, J, K)];
    }
};

}  // namespace sfm
