// Fused per-row stage kernel: the x passes of the demag convolution around every
// effective-field evaluation, with the field terms, the LLG right-hand side and the
// Runge-Kutta stage update in between.
//
// Per block: rpb rows (y, z) x 3 components.
//   A. (fields needed, demag on) load the spectrum rows S1 produced by the y/z passes,
//      undo the packed R2C split, inverse FFT along x  ->  H_demag for the rows (in smem).
//   B. per cell: Heff = Zeeman + H_demag + exchange/iDMI + uniaxial anisotropy,
//      rhs = LLG(M, Heff), then one of: stage update / RKDP54 error estimate / Heff out.
//   C. (forward transform requested) forward FFT along x of the new M rows, R2C split,
//      store to S1 for the next stage's y/z passes.
// Reference physics: Zeeman Boris/Zeeman.cpp:164 (sets Heff, evaluated at the stage time),
// demag Boris/Demag.cpp:170 + Convolution.h:262/659, exchange Boris/Exchange.cpp:108 with
// BorisLib/VEC_VC_Del.h:10, iDMI Boris/iDMExchange.cpp:97 with VEC_VC_Del.h:141 and
// VEC_VC_Grad.h:10,139, anisotropy Boris/Anisotropy.cpp:82, LLG Boris/DiffEqFM_Equations.cpp:12,
// RK4 Boris/DiffEqFM_Evals_RK4.cpp, RKDP54 Boris/DiffEqFM_Evals_RKDP54.cpp, step control
// Boris/DiffEq_CommonBase_Iterate.cpp:15 (SetAdaptiveTimeStep) and :1214 (prime / restore).
#include "kernels.h"
#include "regfft.cuh"

template <typename T>
__device__ __forceinline__ bool stage_gated_out(const StepState *st, int gate)
{
    if (gate == BM_GATE_ALWAYS || st == nullptr) return false;
    if (gate == BM_GATE_ACCEPTED) return *((volatile const int *)&st->reject_flag) != 0;
    return *((volatile const int *)&st->need_restore) == 0;
}

// real value at x of a packed line (complex element x/2, .x for even x, .y for odd x)
template <typename T> __device__ __forceinline__ T *rptr(cpx<T> *line, int x)
{
    return reinterpret_cast<T *>(&line[eaddr<true>(x >> 1, 1)]) + (x & 1);
}

// after a forward complex FFT of z[m] = x[2m] + i x[2m+1]: split into the packed half spectrum
template <typename T>
__device__ __forceinline__ void xfwd_post(cpx<T> *line, int LX, const cpx<T> *__restrict__ tw2, int t, int tpl, bool act)
{
    if (act) {
        for (int k = t; k <= LX / 2; k += tpl) {
            if (k == 0) {
                cpx<T> z0 = line[eaddr<true>(0, 1)];
                line[eaddr<true>(0, 1)] = mk<T>(z0.x + z0.y, z0.x - z0.y);
                continue;
            }
            int k2 = LX - k;
            cpx<T> A = line[eaddr<true>(k, 1)], Bc = conj(line[eaddr<true>(k2, 1)]);
            cpx<T> E = cscale(A + Bc, (T)0.5);
            cpx<T> O = cscale(mul_mi(A - Bc), (T)0.5);
            cpx<T> wO = cmul(tw2[k], O);
            line[eaddr<true>(k, 1)] = E + wO;
            if (k2 != k) line[eaddr<true>(k2, 1)] = conj(E - wO);
        }
    }
    __syncthreads();
}

// inverse of xfwd_post: packed half spectrum -> Z (complex FFT input of the even/odd split)
template <typename T>
__device__ __forceinline__ void xinv_pre(cpx<T> *line, int LX, const cpx<T> *__restrict__ tw2, int t, int tpl, bool act)
{
    if (act) {
        for (int k = t; k <= LX / 2; k += tpl) {
            if (k == 0) {
                cpx<T> p0 = line[eaddr<true>(0, 1)];
                line[eaddr<true>(0, 1)] = mk<T>((p0.x + p0.y) * (T)0.5, (p0.x - p0.y) * (T)0.5);
                continue;
            }
            int k2 = LX - k;
            cpx<T> Xk = line[eaddr<true>(k, 1)], Xk2c = conj(line[eaddr<true>(k2, 1)]);
            cpx<T> E = cscale(Xk + Xk2c, (T)0.5);
            cpx<T> O = cscale(cmul(Xk - Xk2c, conj(tw2[k])), (T)0.5);
            line[eaddr<true>(k, 1)] = E + mul_i(O);
            if (k2 != k) line[eaddr<true>(k2, 1)] = conj(E) + mul_i(conj(O));
        }
    }
    __syncthreads();
}

// versions of xfwd_post / xinv_pre with an element-address functor
template <typename T, typename AddrF>
__device__ __forceinline__ void xfwd_post_f(cpx<T> *line, int LX, const cpx<T> *__restrict__ tw2, int t, int tpl, bool act, AddrF A)
{
    if (act) {
        for (int k = t; k <= LX / 2; k += tpl) {
            if (k == 0) {
                cpx<T> z0 = line[A(0)];
                line[A(0)] = mk<T>(z0.x + z0.y, z0.x - z0.y);
                continue;
            }
            int k2 = LX - k;
            cpx<T> Av = line[A(k)], Bc = conj(line[A(k2)]);
            cpx<T> E = cscale(Av + Bc, (T)0.5);
            cpx<T> O = cscale(mul_mi(Av - Bc), (T)0.5);
            cpx<T> wO = cmul(tw2[k], O);
            line[A(k)] = E + wO;
            if (k2 != k) line[A(k2)] = conj(E - wO);
        }
    }
    __syncthreads();
}

template <typename T, typename AddrF, typename SyncF>
__device__ __forceinline__ void xinv_pre_f(cpx<T> *line, int LX, const cpx<T> *__restrict__ tw2, int t, int tpl, bool act, AddrF A,
                                           SyncF sync)
{
    if (act) {
        for (int k = t; k <= LX / 2; k += tpl) {
            if (k == 0) {
                cpx<T> p0 = line[A(0)];
                line[A(0)] = mk<T>((p0.x + p0.y) * (T)0.5, (p0.x - p0.y) * (T)0.5);
                continue;
            }
            int k2 = LX - k;
            cpx<T> Xk = line[A(k)], Xk2c = conj(line[A(k2)]);
            cpx<T> E = cscale(Xk + Xk2c, (T)0.5);
            cpx<T> O = cscale(cmul(Xk - Xk2c, conj(tw2[k])), (T)0.5);
            line[A(k)] = E + mul_i(O);
            if (k2 != k) line[A(k2)] = conj(E) + mul_i(conj(O));
        }
    }
    sync();
}

template <typename T>
__device__ __forceinline__ void ld3(const T *P, long long n, long long i, T v[3])
{
    v[0] = P[i]; v[1] = P[n + i]; v[2] = P[2 * n + i];
}

// one axis of the Neumann / non-homogeneous Neumann stencils for a full rectangular mesh
// (ih = 1 / h, ih2 = 1 / h^2, products instead of divisions)
template <typename T>
__device__ __forceinline__ void axis_stencil(const T m[3], const T *mp, const T *mm, bool hp, bool hm, T h, T ih, T ih2,
                                             const T bd[3], T d2[3], T g[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (hp && hm) {
            d2[c] = (mp[c] + mm[c] - 2 * m[c]) * ih2;
            g[c] = (mp[c] - mm[c]) * ((T)0.5 * ih);
        } else if (hp) {
            d2[c] = ((mp[c] - m[c]) - bd[c] * h) * ih2;
            g[c] = (T)0.5 * ((mp[c] - m[c]) * ih + bd[c]);
        } else if (hm) {
            d2[c] = ((mm[c] - m[c]) + bd[c] * h) * ih2;
            g[c] = (T)0.5 * ((m[c] - mm[c]) * ih + bd[c]);
        } else {
            d2[c] = 0;
            g[c] = 0;
        }
    }
}

// Per-cell part of a stage: Heff, LLG, update. `lines` holds the 3 * rpb packed x lines of the
// block (component-major), element e of line q at sm[q * LSP + addr(e)]; on entry it carries
// the unscaled inverse-x result (H_demag / scale), on exit the new M (when do_xfwd).
// Per-cell input accessors. AccGlobal reads the device arrays; AccStaged reads the rows the
// register kernel prefetched into shared memory (layout: stage_layout in kernels.h).
template <typename T> struct AccGlobal {
    // pointers copied out of the argument block so each access is (per-cell base)[uniform offset]
    const T *Mn, *Mb, *E[6], *Msm, *K1m;
    long long n, off[5];
    __device__ AccGlobal(const StageArgs<T> &aa) : Mn(aa.Min), Mb(aa.Mbase), Msm(aa.Ms_map), K1m(aa.K1_map), n(aa.n)
    {
#pragma unroll
        for (int i = 0; i < 6; i++) E[i] = aa.ev[i];
        long long nxy = (long long)aa.nx * aa.ny;
        off[0] = 0; off[1] = -aa.nx; off[2] = aa.nx; off[3] = -nxy; off[4] = nxy;
    }
    __device__ __forceinline__ T m(int, int slot, int c, int, long long cell) const { return (Mn + cell)[c * n + off[slot]]; }
    __device__ __forceinline__ T mb(int, int c, int, long long cell) const { return (Mb + cell)[c * n]; }
    __device__ __forceinline__ T ev(int i, int, int c, int, long long cell) const { return (E[i] + cell)[c * n]; }
    __device__ __forceinline__ T ms(int, int, long long cell) const { return Msm[cell]; }
    __device__ __forceinline__ T k1(int, int, long long cell) const { return K1m[cell]; }
};

template <typename T> struct AccStaged {
    const T *R;
    int nx, kr, ns3, hasmb, evo, mso, k1o;
    __device__ __forceinline__ const T *row(int r, int k) const { return R + ((long long)r * kr + k) * nx; }
    __device__ __forceinline__ T m(int r, int slot, int c, int x, long long) const { return row(r, slot * 3 + c)[x]; }
    __device__ __forceinline__ T mb(int r, int c, int x, long long) const { return row(r, hasmb ? ns3 + c : c)[x]; }
    __device__ __forceinline__ T ev(int i, int r, int c, int x, long long) const { return row(r, evo + 3 * i + c)[x]; }
    __device__ __forceinline__ T ms(int r, int x, long long) const { return row(r, mso)[x]; }
    __device__ __forceinline__ T k1(int r, int x, long long) const { return row(r, k1o)[x]; }
};

// sum[c] += sum_{i < NEV} cev[i] * ev_i[c] (component by component, i ascending)
template <int NEV, typename T, typename Acc>
__device__ __forceinline__ void ev_acc(const Acc &acc, const T *cev, int r, int x, long long cell, T sum[3])
{
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int i = 0; i < NEV; i++) sum[c] += cev[i] * acc.ev(i, r, c, x, cell);
}

// sum_{i < NEV} c1[i] * ev_i[c] and sum_{i < NEV} c2[i] * ev_i[c] in FP64, i ascending, each ev_i
// loaded once (the RKDP54 error estimate's 4th-order prediction and embedded 5th-order solution)
template <int NEV, typename Acc>
__device__ __forceinline__ void ev_sum2_d(const Acc &acc, const double *c1, const double *c2, int r, int c, int x,
                                          long long cell, double &s1, double &s2)
{
    double a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int i = 0; i < NEV; i++) {
        const double e = (double)acc.ev(i, r, c, x, cell);
        a1 += c1[i] * e;
        a2 += c2[i] * e;
    }
    s1 = a1;
    s2 = a2;
}

// sum_{i < NEV} cev[i] * ev_i[c] in FP64 (error estimate)
template <int NEV, typename Acc>
__device__ __forceinline__ double ev_sum_d(const Acc &acc, const double *cev, int r, int c, int x, long long cell)
{
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < NEV; i++) sum += cev[i] * (double)acc.ev(i, r, c, x, cell);
    return sum;
}

// Per-block maxima of the torque and dm/dt diagnostics (non-negative doubles as bits)
__device__ __forceinline__ unsigned long long *stage_diag_slots()
{
    __shared__ unsigned long long slots[2];
    return slots;
}

// the BM_DIAG_MXH / BM_DIAG_DMDT bits of this launch that the host requested (the request stays set
// until the last block of the set's publishing launch clears it, so every block reads the same)
template <typename T> __device__ __forceinline__ int stage_diag_active(const StageArgs<T> &a)
{
    if (!a.diag || !a.st) return 0;
    int d = 0;
    if ((a.diag & BM_DIAG_MXH) && *((volatile const int *)&a.st->calc_mxh)) d |= BM_DIAG_MXH;
    if ((a.diag & BM_DIAG_DMDT) && *((volatile const int *)&a.st->calc_dmdt)) d |= BM_DIAG_DMDT;
    return d;
}

// SPEC 1: the plain stage update (stage_plain on the host): mode, the outputs written and the demag
// and exchange terms are compile-time, so their run-time checks leave the per-cell loop; SPEC 2 the
// plain RKDP54 error estimate (stage_lte_plain), SPEC 3 the plain advance of the base state
// (stage_adv_plain), likewise
template <typename T, int SPEC = 0, typename AddrF, typename Acc>
__device__ __forceinline__ void stage_cells(const StageArgs<T> &a, cpx<T> *sm, int LSP, AddrF addr, int r0, double &lmax,
                                            const Acc &acc)
{
    constexpr bool PS = SPEC == 1, PL = SPEC == 2, PA = SPEC == 3, SP = SPEC != 0;
    const int nx = a.nx, ny = a.ny, nz = a.nz, rpb = a.rpb;
    const int nrows = ny * nz;
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long n = a.n;
    const int mode = PS ? BM_MODE_STAGE : PL ? BM_MODE_LTE : PA ? BM_MODE_UPDATE : a.mode;
    const T *Hd = SP ? nullptr : a.Hd;
    T *Hsave = SP ? nullptr : a.Hsave;
    T *Ysave = SP ? nullptr : a.Ysave;
    T *copy_to = (PS || PL) ? nullptr : a.copy_to;
    const bool has_ev_out = (PS || PL) || (!PA && a.ev_out), has_Mout = (PS || PA) || (!PL && a.Mout);
    const bool do_xfwd = (PS || PA) || (!PL && a.do_xfwd);
    const bool fields = (PS || PL) || (!PA && mode != BM_MODE_UPDATE);
    const bool demag = (PS || PL) || (!PA && fields && (a.modules & BM_MOD_DEMAG));
    const double dT = a.st ? *((volatile double *)&a.st->dT) : 0.0;
    T Ha[3] = {0, 0, 0};
    if (fields && (a.modules & BM_MOD_ZEEMAN) && a.Ha && a.nHa > 0) {
        double tm = a.st ? *((volatile double *)&a.st->stagetime) : 0.0;
        int hi = 0;
        if (a.nHa > 1 && a.Ha_tspan > 0.0) {
            // one FP64 division per warp, broadcast (every launch runs whole warps)
            if ((threadIdx.x & 31) == 0) {
                hi = (int)floor(tm / a.Ha_tspan * a.nHa);
                hi = hi < 0 ? 0 : (hi >= a.nHa ? a.nHa - 1 : hi);
            }
            hi = __shfl_sync(0xffffffffu, hi, 0);
        }
        Ha[0] = (T)a.Ha[3 * hi]; Ha[1] = (T)a.Ha[3 * hi + 1]; Ha[2] = (T)a.Ha[3 * hi + 2];
    }
    const bool exch = (PS || PL) || (!PA && fields && (a.modules & (BM_MOD_EXCH | BM_MOD_IDMI)));
    const bool idmi = (a.modules & BM_MOD_IDMI) != 0;
    const bool zflat = (nz == 1);
    // torque / dm/dt diagnostics of this launch (meshes with grel = 0 take no part, as in the
    // reference's reductions)
    const int dg = (a.grel != (T)0) ? stage_diag_active(a) : 0;
    unsigned long long *dslot = stage_diag_slots();
    if (stage_diag_active(a)) {
        if (tid == 0) { dslot[0] = 0ull; dslot[1] = 0ull; }
        __syncthreads();
    }
    const int nev = a.nev;
    T cev[6];
#pragma unroll
    for (int i = 0; i < 6; i++) cev[i] = (T)(a.cev[i] * dT);
    const T crhs = (T)(a.crhs * dT);
    const int cstride = 2 * rpb * LSP;   // T elements between the component lines of one row
    // (r, x) of cell index ci = r * nx + x, advanced by nt per iteration without divisions
    int dr = 0, dx = nt, r = 0, x = tid;   // a block no wider than a row: no divisions
    if (nt > nx) {
        dr = nt / nx; dx = nt - dr * nx;
        r = tid / nx; x = tid - r * nx;
    }
    // one cell (r, x) of the block's rows at (y, z): fields, LLG rhs, stage update and outputs
    auto cell_body = [&](int r, int x, int y, int z, long long cell) {
        T *sp = reinterpret_cast<T *>(&sm[r * LSP + addr(x >> 1)]) + (x & 1);   // packed line slot of x
        T m[3];
#pragma unroll
        for (int c = 0; c < 3; c++) m[c] = acc.m(r, 0, c, x, cell);
        const T Ms = a.Ms_map ? acc.ms(r, x, cell) : a.Ms;
        const T iMs = a.Ms_map ? (T)1 / Ms : a.iMs;
        T rhs[3] = {0, 0, 0};
        if (fields) {
            T H[3] = {Ha[0], Ha[1], Ha[2]};
            if (demag) {
#pragma unroll
                for (int c = 0; c < 3; c++) H[c] += a.scale * sp[c * cstride];
            }
            if (Hd) {
#pragma unroll
                for (int c = 0; c < 3; c++) H[c] += (Hd + cell)[c * n];
            }
            const bool hxp = x + 1 < nx, hxm = x > 0, hyp = y + 1 < ny, hym = y > 0, hzp = z + 1 < nz, hzm = z > 0;
            if (exch && hxp && hxm && hyp && hym && (zflat || (hzp && hzm))) {
                // interior cell: both neighbours on every axis (the first branch of axis_stencil;
                // a one-cell-thick mesh has no z terms)
                const T iMs2 = iMs * iMs;
                const T Ac = a.exA * iMs2;
                T lap[3], gxv[3], gyv[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const T mxp = acc.m(r, 0, c, x + 1, cell + 1), mxm = acc.m(r, 0, c, x - 1, cell - 1);
                    const T mym = acc.m(r, 1, c, x, cell), myp = acc.m(r, 2, c, x, cell);
                    const T dx2 = (mxp + mxm - 2 * m[c]) * a.ih2[0];
                    const T dy2 = (myp + mym - 2 * m[c]) * a.ih2[1];
                    T dz2 = 0;
                    if (!zflat) {
                        const T mzm = acc.m(r, 3, c, x, cell), mzp = acc.m(r, 4, c, x, cell);
                        dz2 = (mzp + mzm - 2 * m[c]) * a.ih2[2];
                    }
                    lap[c] = dx2 + dy2 + dz2;
                    gxv[c] = (mxp - mxm) * ((T)0.5 * a.ih[0]);
                    gyv[c] = (myp - mym) * ((T)0.5 * a.ih[1]);
                }
                if (idmi) {
                    const T Dc = a.exD * iMs2;
                    const T hd[3] = {gxv[2], gyv[2], -gxv[0] - gyv[1]};
#pragma unroll
                    for (int c = 0; c < 3; c++) H[c] += Ac * lap[c] + Dc * hd[c];
                } else {
#pragma unroll
                    for (int c = 0; c < 3; c++) H[c] += Ac * lap[c];
                }
            } else if (exch) {
                T mxp[3], mxm[3], myp[3], mym[3], mzp[3], mzm[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    mxp[c] = hxp ? acc.m(r, 0, c, x + 1, cell + 1) : (T)0;
                    mxm[c] = hxm ? acc.m(r, 0, c, x - 1, cell - 1) : (T)0;
                    mym[c] = hym ? acc.m(r, 1, c, x, cell) : (T)0;
                    myp[c] = hyp ? acc.m(r, 2, c, x, cell) : (T)0;
                    mzm[c] = hzm ? acc.m(r, 3, c, x, cell) : (T)0;
                    mzp[c] = hzp ? acc.m(r, 4, c, x, cell) : (T)0;
                }
                // periodic axes: the missing neighbour is the cell on the far side, times the axis'
                // sign (the PBC branch of delsq_nneu / grad_nneu, BorisLib/VEC_VC_Del.h:141,
                // BorisLib/VEC_VC_Grad.h:139); a one-cell axis has no neighbours either way
                bool bxp = hxp, bxm = hxm, byp = hyp, bym = hym, bzp = hzp, bzm = hzm;
                if (a.pbc[0] && nx > 1) {
                    const T sg = (T)a.pbc[0];
                    if (!hxp) { bxp = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) mxp[c] = sg * acc.m(r, 0, c, 0, cell - (nx - 1)); }
                    if (!hxm) { bxm = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) mxm[c] = sg * acc.m(r, 0, c, nx - 1, cell + (nx - 1)); }
                }
                if (a.pbc[1] && ny > 1) {
                    const T sg = (T)a.pbc[1];
                    const long long w = (long long)(ny - 1) * nx;
                    if (!hyp) { byp = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) myp[c] = sg * (a.Min + (cell - w))[c * n]; }
                    if (!hym) { bym = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) mym[c] = sg * (a.Min + (cell + w))[c * n]; }
                }
                if (a.pbc[2] && nz > 1) {
                    const T sg = (T)a.pbc[2];
                    const long long w = (long long)(nz - 1) * nx * ny;
                    if (!hzp) { bzp = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) mzp[c] = sg * (a.Min + (cell - w))[c * n]; }
                    if (!hzm) { bzm = true;
#pragma unroll
                        for (int c = 0; c < 3; c++) mzm[c] = sg * (a.Min + (cell + w))[c * n]; }
                }
                const T rr = idmi ? a.rrD : (T)0;
                T bx[3] = {rr * m[2], 0, -rr * m[0]};
                T by[3] = {0, rr * m[2], -rr * m[1]};
                T bz[3] = {0, 0, 0};
                T dx2[3], dy2[3], dz2[3], gx[3], gy[3], gz[3];
                axis_stencil<T>(m, mxp, mxm, bxp, bxm, a.hh[0], a.ih[0], a.ih2[0], bx, dx2, gx);
                axis_stencil<T>(m, myp, mym, byp, bym, a.hh[1], a.ih[1], a.ih2[1], by, dy2, gy);
                axis_stencil<T>(m, mzp, mzm, bzp, bzm, a.hh[2], a.ih[2], a.ih2[2], bz, dz2, gz);
                const T iMs2 = iMs * iMs;
                const T Ac = a.exA * iMs2;
                const T Dc = idmi ? a.exD * iMs2 : (T)0;
                T hd[3] = {gx[2], gy[2], -gx[0] - gy[1]};
#pragma unroll
                for (int c = 0; c < 3; c++) H[c] += Ac * (dx2[c] + dy2[c] + dz2[c]) + Dc * hd[c];
            }
            if (a.modules & BM_MOD_ANIUNI) {
                T K1 = a.K1_map ? acc.k1(r, x, cell) : a.K1;
                T dp = (m[0] * a.ea[0] + m[1] * a.ea[1] + m[2] * a.ea[2]) * iMs;
                T s = (a.two_mu0 * iMs) * dp * (K1 + 2 * a.K2 * (1 - dp * dp));
#pragma unroll
                for (int c = 0; c < 3; c++) H[c] += s * a.ea[c];
            }
            if (mode == BM_MODE_HEFF) {
#pragma unroll
                for (int c = 0; c < 3; c++) (a.Hout + cell)[c * n] = H[c];
                return;
            }
            if (Hsave) {
#pragma unroll
                for (int c = 0; c < 3; c++) (Hsave + cell)[c * n] = H[c];
            }
            T mxh[3] = {m[1] * H[2] - m[2] * H[1], m[2] * H[0] - m[0] * H[2], m[0] * H[1] - m[1] * H[0]};
            if (dg & BM_DIAG_MXH) {
                // |M x Heff| / |M|^2 (DiffEqFM_EvalsCUDA_RKDP54.cu:31-32, DiffEqFM_EvalsLLGCUDA.cu:445-446),
                // in the stage's precision as the reference's reduction kernels compute it
                const T x2 = mxh[0] * mxh[0] + mxh[1] * mxh[1] + mxh[2] * mxh[2];
                const T m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                atomicMax(&dslot[0], (unsigned long long)__double_as_longlong((double)(sqrt(x2) / m2)));
            }
            T mu[3] = {m[0] * iMs, m[1] * iMs, m[2] * iMs};
            T mmxh[3] = {mu[1] * mxh[2] - mu[2] * mxh[1], mu[2] * mxh[0] - mu[0] * mxh[2], mu[0] * mxh[1] - mu[1] * mxh[0]};
#pragma unroll
            for (int c = 0; c < 3; c++) rhs[c] = a.llg_pre * (mxh[c] + a.alpha * mmxh[c]);
        }
        if (mode == BM_MODE_LTE) {
            // 4th-order prediction from the previous step's stages (FSAL), error in FP64
            double d2 = 0.0, m2 = 0.0;
            double sb[3], sa[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                sb[c] = 0.0;
                sa[c] = 0.0;
                if (a.lte_embedded && nev == 5) {
                    // both weightings of the five stage evaluations from one load of each
                    ev_sum2_d<5>(acc, a.cev, a.cev5, r, c, x, cell, sb[c], sa[c]);
                    continue;
                }
                switch (nev) {   // block-uniform: unrolled sums without predicated loads
                case 6: sb[c] = ev_sum_d<6>(acc, a.cev, r, c, x, cell); break;
                case 5: sb[c] = ev_sum_d<5>(acc, a.cev, r, c, x, cell); break;
                case 4: sb[c] = ev_sum_d<4>(acc, a.cev, r, c, x, cell); break;
                case 3: sb[c] = ev_sum_d<3>(acc, a.cev, r, c, x, cell); break;
                case 2: sb[c] = ev_sum_d<2>(acc, a.cev, r, c, x, cell); break;
                case 1: sb[c] = ev_sum_d<1>(acc, a.cev, r, c, x, cell); break;
                default: break;
                }
            }
            if (a.lte_embedded) {
                // the step's 5th-order solution recomputed in FP64 from its base and stage rhs,
                // renormalised to Ms, against the 4th-order prediction: the reference's
                // |M - prediction| without the rounding of the FP32-stored M
                double m5[3], n5 = 0.0;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    m5[c] = (double)acc.mb(r, c, x, cell) + dT * sa[c];
                    n5 += m5[c] * m5[c];
                }
                const double f = (double)Ms / sqrt(n5);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double pred = (double)acc.mb(r, c, x, cell) + dT * (sb[c] + a.crhs * (double)rhs[c]);
                    const double d = m5[c] * f - pred;
                    d2 += d * d;
                    m2 += (double)m[c] * (double)m[c];
                }
            } else {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double pred = (double)acc.mb(r, c, x, cell) + dT * (sb[c] + a.crhs * (double)rhs[c]);
                    const double d = (double)m[c] - pred;
                    d2 += d * d;
                    m2 += (double)m[c] * (double)m[c];
                }
            }
            // a non-finite current state (M or its rhs) is flagged, never accepted; a NaN error
            // estimate from the stage buffers of an unprimed attempt only counts as a huge error
            if (!isfinite(m[0] + m[1] + m[2] + rhs[0] + rhs[1] + rhs[2])) atomicOr(&a.st->error, BM_ERR_NONFINITE);
            double l = sqrt(d2) / sqrt(m2);
            if (!(l <= 1e300)) l = 1e300;
            if (l > lmax) lmax = l;
#pragma unroll
            for (int c = 0; c < 3; c++) (a.ev_out + cell)[c * n] = rhs[c];
            return;
        }
        T mn[3];
        {
            T sum[3] = {crhs * rhs[0], crhs * rhs[1], crhs * rhs[2]};
            switch (nev) {   // block-uniform: unrolled sums without predicated loads
            case 6: ev_acc<6>(acc, cev, r, x, cell, sum); break;
            case 5: ev_acc<5>(acc, cev, r, x, cell, sum); break;
            case 4: ev_acc<4>(acc, cev, r, x, cell, sum); break;
            case 3: ev_acc<3>(acc, cev, r, x, cell, sum); break;
            case 2: ev_acc<2>(acc, cev, r, x, cell, sum); break;
            case 1: ev_acc<1>(acc, cev, r, x, cell, sum); break;
            default: break;
            }
#pragma unroll
            for (int c = 0; c < 3; c++) mn[c] = acc.mb(r, c, x, cell) + sum[c];
        }
        if (Ysave) {
#pragma unroll
            for (int c = 0; c < 3; c++) (Ysave + cell)[c * n] = mn[c];
        }
        if (!PA && a.renorm) {
            T f = Ms / sqrt(mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2]);
            mn[0] *= f; mn[1] *= f; mn[2] *= f;
            // the step's new state must be finite (the sum is non-finite if any component is)
            if (!isfinite(mn[0] + mn[1] + mn[2]) && a.st) atomicOr(&a.st->error, BM_ERR_NONFINITE);
        }
        if (dg & BM_DIAG_DMDT) {
            // |M - M_start| / (dT GAMMA |M|^2) after the last stage (DiffEqFM_EvalsLLGCUDA.cu:583-584,
            // DiffEqFM_EvalsCUDA_RKDP54.cu:216-217); the step base is read before this cell's M is written
            T d2 = 0, m2 = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const T d = mn[c] - acc.mb(r, c, x, cell);
                d2 += d * d;
                m2 += mn[c] * mn[c];
            }
            atomicMax(&dslot[1], (unsigned long long)__double_as_longlong((double)sqrt(d2) / (dT * BM_GAMMA * (double)m2)));
        }
        if (has_ev_out) {
#pragma unroll
            for (int c = 0; c < 3; c++) (a.ev_out + cell)[c * n] = rhs[c];
        }
        if (copy_to) {
#pragma unroll
            for (int c = 0; c < 3; c++) (copy_to + cell)[c * n] = m[c];
        }
        if (has_Mout) {
#pragma unroll
            for (int c = 0; c < 3; c++) (a.Mout + cell)[c * n] = mn[c];
        }
        if (do_xfwd) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                sp[c * cstride] = mn[c];
                if ((x & 1) == 0 && x == nx - 1) sp[c * cstride + 1] = 0;   // odd nx: zero the partner slot
            }
        }
    };
    int yrow = -1, y = 0, z = 0;
    for (; r < rpb; x += dx, r += dr) {
        if (x >= nx) { x -= nx; r++; if (r >= rpb) break; }
        const int row = r0 + r;
        if (row >= nrows) break;
        if (row != yrow) { yrow = row; z = row / ny; y = row - z * ny; }
        cell_body(r, x, y, z, (long long)row * nx + x);
    }
}

// LTE block reduction and the last-block bookkeeping (step finish / controller / restore flag)
// total: launch items that each call the tail once (blocks, or work items of a batched launch)
template <typename T, int SPEC = 0>
__device__ __forceinline__ void stage_tail(const StageArgs<T> &a, double lmax, unsigned int total)
{
    __shared__ double red[32];
    __shared__ int is_last;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (SPEC == 2 || (SPEC == 0 && a.mode == BM_MODE_LTE)) {
        for (int o = 16; o > 0; o >>= 1) {
            double v = __shfl_xor_sync(0xffffffffu, lmax, o);
            if (v > lmax) lmax = v;
        }
        if ((tid & 31) == 0) red[tid >> 5] = lmax;
        __syncthreads();
        if (tid == 0) {
            double b = 0.0;
            for (int w = 0; w < (nt + 31) / 32; w++) if (red[w] > b) b = red[w];
            atomicMax(&a.st->lte_bits, (unsigned long long)__double_as_longlong(b));
        }
    }
    const int dg = stage_diag_active(a);
    if (dg) {
        // the block's diagnostic maxima into the running maxima of the set
        __syncthreads();
        if (tid == 0) {
            const unsigned long long *dslot = stage_diag_slots();
            if (dg & BM_DIAG_MXH) atomicMax(&a.st->mxh_acc, dslot[0]);
            if (dg & BM_DIAG_DMDT) atomicMax(&a.st->dmdt_acc, dslot[1]);
        }
    }
    const bool publish = dg && (a.diag & BM_DIAG_PUBLISH);
    if ((a.last_kind == BM_LAST_NONE && !publish) || a.st == nullptr) return;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        unsigned int tk = atomicAdd(&a.st->blocks_done, 1u);
        is_last = (tk == total - 1);
    }
    __syncthreads();
    if (!is_last || tid != 0) return;
    __threadfence();
    volatile StepState *st = a.st;
    if (publish) {
        // the set's maxima become the values Get_mxh / Get_dmdt return; the request is served
        if (dg & BM_DIAG_MXH) {
            st->mxh = __longlong_as_double((long long)atomicExch(&a.st->mxh_acc, 0ull));
            st->calc_mxh = 0;
        }
        if (dg & BM_DIAG_DMDT) {
            st->dmdt = __longlong_as_double((long long)atomicExch(&a.st->dmdt_acc, 0ull));
            st->calc_dmdt = 0;
        }
    }
    if (a.last_kind == BM_LAST_FINISH) {
        st->time = st->time + st->dT;
        st->stagetime = st->stagetime + st->dT;
        st->accepted = st->accepted + 1;
        st->es_available = 1;   // the step completed (the reference's `available`)
    } else if (a.last_kind == BM_LAST_RESTORED) {
        st->need_restore = 0;
    } else if (a.last_kind == BM_LAST_CONTROL) {
        double lte = __longlong_as_double((long long)atomicAdd(&a.st->lte_bits, 0ull));
        st->attempts = st->attempts + 1;
        st->reject_flag = 0;
        if (st->error) {
            // a non-finite state: the step that produced it is taken back (restored at the next
            // attempt) and the rest of this attempt is skipped, whatever dT is; the host stops
            if (st->primed) {
                st->time = st->time - st->dT;
                st->stagetime = st->stagetime - st->dT;
                st->accepted = st->accepted - 1;
                st->rejected = st->rejected + 1;
                st->need_restore = 1;
                st->es_available = 0;
            }
            st->primed = 0;
            st->reject_flag = 1;
        } else if (!st->primed) {
            st->primed = 1;
        } else {
            st->dT_last = st->dT;
            st->last_lte = lte;
            st->lte = lte;
            double tol = st->tol, dT = st->dT, dmin = st->dT_min, dmax = st->dT_max;
            double ord = (double)(st->eval_order + 1);
            if (dmin != dmax) {
                if (lte > tol && dT > dmin) {
                    st->es_available = 0;   // failed, must repeat (SetAdaptiveTimeStep)
                    st->time = st->time - dT;
                    st->stagetime = st->stagetime - dT;
                    st->accepted = st->accepted - 1;
                    st->rejected = st->rejected + 1;
                    double c = pow(tol * 0.8 / lte, 1.0 / ord);
                    if (c < 0.01) c = 0.01;
                    dT *= c;
                    if (dT < dmin) dT = dmin;
                    st->dT = dT;
                    st->reject_flag = 1;
                    st->need_restore = 1;
                    st->primed = 0;
                } else if (lte > 0) {
                    double c = pow(tol * 0.8 / lte, 1.0 / ord);
                    if (c > st->dT_incr) c = st->dT_incr;
                    if (c < 0.01) c = 0.01;
                    dT *= c;
                    if (dT < dmin) dT = dmin;
                    if (dT > dmax) dT = dmax;
                    st->dT = dT;
                }
            }
        }
    }
    st->lte_bits = 0ull;
    st->blocks_done = 0u;
    __threadfence();
}

// generic-length body (shared-memory Stockham x transforms) for row block bid
template <typename T>
__device__ __forceinline__ void stage_generic_body(const StageArgs<T> &a, int bid, unsigned int total)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    const int LX = a.LX, rpb = a.rpb, tpl = a.px.tpl;
    const int LSP = padded_len(LX);
    const int nrows = a.ny * a.nz;
    const int r0 = bid * rpb;
    const int tid = threadIdx.x;
    const int q = tid / tpl, t = tid % tpl;
    const int qc = q / rpb, qr = q % rpb;
    const bool qact = (q < 3 * rpb) && (r0 + qr < nrows);
    cpx<T> *line = sm + (q < 3 * rpb ? q : 0) * LSP;
    const bool demag = (a.mode != BM_MODE_UPDATE) && (a.modules & BM_MOD_DEMAG);
    if (demag) {
        if (qact) {
            const cpx<T> *src = a.S1 + ((long long)qc * nrows + r0 + qr) * LX;
            for (int m = t; m < LX; m += tpl) cp_async_cpx<T>(&line[eaddr<true>(m, 1)], &src[m], true);
        }
        cp_async_wait_all();
        __syncthreads();
        xinv_pre<T>(line, LX, a.twx2, t, tpl, qact);
        fft_line<T, true, true>(line, 1, t, qact, a.px, a.twx);
    }
    double lmax = 0.0;
    stage_cells<T>(a, sm, LSP, [](int e) { return eaddr<true>(e, 1); }, r0, lmax, AccGlobal<T>(a));
    if (a.do_xfwd) {
        const int first_pad = (a.nx + 1) >> 1;
        for (int idx = tid; idx < 3 * rpb * LX; idx += blockDim.x) {
            int qq = idx / LX, mm = idx - qq * LX;
            if (mm >= first_pad) sm[qq * LSP + eaddr<true>(mm, 1)] = mk<T>(0, 0);
        }
        __syncthreads();
        fft_line<T, true, false>(line, 1, t, qact, a.px, a.twx);
        xfwd_post<T>(line, LX, a.twx2, t, tpl, qact);
        if (qact) {
            cpx<T> *dst = a.S1 + ((long long)qc * nrows + r0 + qr) * LX;
            for (int mm = t; mm < LX; mm += tpl) dst[mm] = line[eaddr<true>(mm, 1)];
        }
    }
    stage_tail<T>(a, lmax, total);
}

template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_stage(StageArgs<T> a)
{
    if (stage_gated_out<T>(a.st, a.gate)) return;
    stage_generic_body<T>(a, blockIdx.x, gridDim.x);
}

// many meshes in one launch: work item (mesh, row block). The meshes share the step state; every
// item takes part in the error-norm maximum and the last item finishes the step (last_kind is the
// same for all meshes of the launch).
template <typename T>
__global__ void __launch_bounds__(bm_lb<T>::v) k_stage_batch(const StageArgs<T> *__restrict__ args, const int2 *__restrict__ work,
                                                                int nwork)
{
    if (stage_gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    stage_generic_body<T>(args[it.x], it.y, (unsigned int)nwork);
}

// ---------------------------------------------------------------------------------------------
// Register kernels for power-of-two LX (16 .. 1024). Two x-transform variants:
//   xv 0: LX = P * Q (P <= Q <= 32): one DFT_Q and one DFT_P per thread in registers around one
//         shared transpose (line padded one slot per P elements, so both access patterns are
//         conflict-free); Q threads per line.
//   xv 1: radix-8 Stockham (the last pass takes the remaining radix 2 or 4), LX / 8 threads per
//         line each holding 8 values per pass, line padded one slot per 16 elements; compiled
//         with a register cap (64 FP32, 128 FP64) so that more rows are resident per SM.
// The packed-spectrum split (xinv_pre / xfwd_post) and the per-cell work stay in shared memory
// in natural order.
// register cap of the FP32 Stockham stage kernels (more resident rows per SM against spills)
#ifndef BM_RX_MAXNREG_F
#define BM_RX_MAXNREG_F 64
#endif
// xv 3: the radix-16 kernel of xv 2 at a lower FP32 cap (12 instead of 10 resident 96-thread
// blocks per SM, more spills); the autotuner times both
#ifndef BM_RX16_LO_MAXNREG_F
#define BM_RX16_LO_MAXNREG_F 56
#endif

template <int P> struct addrP {
    __device__ __forceinline__ int operator()(int e) const { return e + e / P; }
};

template <int LX> struct xr_pq {
    static constexpr int P = LX == 16 ? 4 : LX == 32 ? 4 : LX == 64 ? 8 : LX == 128 ? 8 : LX == 256 ? 16 : LX == 512 ? 16 : 32;
    static constexpr int Q = LX / P;
};

// Stockham shape: power-of-two L, 8 values per thread (radix 8, the last pass the remaining 2 or
// 4); L = 3 * 2^k, 12 values per thread (radix 4, one radix 2 where the power of two is odd, then
// the radix-3 pass last so that every earlier stride is a power of two)
// (VW = 16: the radix-16 variant of the power-of-two shape, 16 values per thread and half the
// threads per line, so each thread carries twice the cells of the per-cell phase)
template <int L, int VW = 8> struct xs_shape {
    static constexpr int V = (L % 3 == 0) ? 12 : VW;
    static constexpr int TPL = L / V;
};
template <int L, int NS, int VW = 8> struct xs_radix {
    static constexpr int M = L / NS;
    static constexpr int v = (L % 3) ? (M >= VW ? VW : M) : ((M % 4 == 0 && M / 4 >= 3) ? 4 : (M % 2 == 0 && M / 2 >= 3) ? 2 : 3);
};

template <int LX, int XV> struct xr_cfg {
    static constexpr int PAD = XV == 0 ? xr_pq<LX>::P : 16;   // one padding slot per PAD elements
    static constexpr int TPL = XV == 0 ? xr_pq<LX>::Q : xs_shape<LX, XV == 2 ? 16 : 8>::TPL;   // threads per line
    static constexpr int LSP = LX + LX / PAD + 1;             // padded line length
};

template <typename T, int P, int Q, bool INV>
__device__ __forceinline__ void x_twolevel(cpx<T> *line, int t, bool act, const cpx<T> *__restrict__ tw, int nkeep)
{
    addrP<P> A;
    cpx<T> v[Q];
    if (act && t < P) {
#pragma unroll
        for (int n2 = 0; n2 < Q; n2++) {
            if (!INV && n2 >= Q / 2) v[n2] = mk<T>(0, 0);   // forward input is zero beyond LX/2
            else v[n2] = line[A(t + P * n2)];
        }
    }
    __syncthreads();
    if (act && t < P) {
        RegFFT<T, Q, INV>::run(v, tw, P);
#pragma unroll
        for (int k2 = 0; k2 < Q; k2++) {
            cpx<T> x = v[k2];
            if (k2 > 0 && t > 0) {
                cpx<T> w = tw[t * k2];
                if (INV) w.y = -w.y;
                x = cmul(x, w);
            }
            line[A(k2 * P + t)] = x;
        }
    }
    __syncthreads();
    cpx<T> u[P];
    if (act && t < Q) {
#pragma unroll
        for (int n1 = 0; n1 < P; n1++) u[n1] = line[A(t * P + n1)];
    }
    __syncthreads();
    if (act && t < Q) {
        RegFFT<T, P, INV>::run(u, tw, Q);
#pragma unroll
        for (int k1 = 0; k1 < P; k1++) {
            const int e = t + Q * k1;
            if (!INV || e < nkeep) line[A(e)] = u[k1];
        }
    }
    __syncthreads();
}

// Barrier between the radix passes of x lines: where the threads of a line divide a warp (and the
// block is whole warps), every warp owns whole lines and synchronises alone; otherwise the block.
template <int TPL> __device__ __forceinline__ void xs_sync()
{
    if constexpr (32 % TPL == 0) {
        if ((blockDim.x & 31) == 0) {
            __syncwarp();
            return;
        }
    }
    __syncthreads();
}

// One Stockham pass of stride NS (radix R from xs_radix) and the passes after it. Butterfly j
// reads elements j + r * L / R, twiddles them by w_L^(r k L / (NS R)) (k = j mod NS), and writes
// the R-point DFT to (j - k) R + k + r NS. ZHALF: the input is zero beyond L / 2 (only the first
// pass reads it: there element j + r L / R >= L / 2 exactly when r >= R / 2). The last inverse
// pass stores only elements below nkeep.
template <typename T, int L, int NS, bool INV, bool ZHALF, int VW = 8>
__device__ __forceinline__ void x_stockham(cpx<T> *line, int t, bool act, const cpx<T> *__restrict__ tw, int nkeep)
{
    constexpr int TPL = xs_shape<L, VW>::TPL;
    constexpr int R = xs_radix<L, NS, VW>::v;
    constexpr int LR = L / R, BPT = LR / TPL, TWS = L / (NS * R);
    constexpr bool LAST = NS * R == L;
    addrP<16> A;
    // padded addresses: A(e + 16 q) = A(e) + 17 q, so strides that are multiples of 16 become
    // compile-time offsets from one runtime base
    constexpr bool LRP = (LR % 16) == 0, TPP = (TPL % 16) == 0, NSP = (NS % 16) == 0;
    cpx<T> v[BPT][R];
    if (act) {
        const int at = A(t);
#pragma unroll
        for (int b = 0; b < BPT; b++) {
            const int ab = TPP ? at + b * (TPL + TPL / 16) : A(t + b * TPL);
#pragma unroll
            for (int r = 0; r < R; r++) {
                if (ZHALF && 2 * r >= R) v[b][r] = mk<T>(0, 0);
                else v[b][r] = line[LRP ? ab + r * (LR + LR / 16) : A(t + b * TPL + r * LR)];
            }
        }
    }
    xs_sync<TPL>();
    if (act) {
#pragma unroll
        for (int b = 0; b < BPT; b++) {
            const int j = t + b * TPL;
            const int k = j & (NS - 1);
            if (NS > 1) {
                const int step = k * TWS;
                const cpx<T> *tp = tw;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    tp += step;
                    cpx<T> w = *tp;
                    if (INV) w.y = -w.y;
                    v[b][r] = cmul(v[b][r], w);
                }
            }
            dftR<T, R, INV>(v[b]);
            const int d = (j - k) * R + k;
            const int ad = A(d);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int e = d + r * NS;
                if (!INV || !LAST || e < nkeep) line[NSP ? ad + r * (NS + NS / 16) : A(e)] = v[b][r];
            }
        }
    }
    xs_sync<TPL>();
    if constexpr (!LAST) x_stockham<T, L, NS * R, INV, false, VW>(line, t, act, tw, nkeep);
}

template <typename T, int LX, int XV, bool INV>
__device__ __forceinline__ void x_reg(cpx<T> *line, int t, bool act, const cpx<T> *__restrict__ tw, int nkeep)
{
    if constexpr (XV == 0) x_twolevel<T, xr_pq<LX>::P, xr_pq<LX>::Q, INV>(line, t, act, tw, nkeep);
    else if constexpr (XV == 1) x_stockham<T, LX, 1, INV, !INV>(line, t, act, tw, nkeep);
    else x_stockham<T, LX, 1, INV, !INV, 16>(line, t, act, tw, nkeep);
}

// The evaluation speedup's extrapolation on one x line in shared memory (element e at line[A(e)]):
// es_cs[c] line + sum_k a_k G_k[c][row] (the sum of k_es_extrap), when this evaluation extrapolates:
// RK4 (es_fold 1) once es_K fields are saved, RKDP54 (es_fold 2) when the decision says so.
template <typename T, int LX, int PAD>
__device__ __noinline__ void es_fold_line(const StepState *st, int fold, const cpx<T> *esG, T f, double ceval, int nrows,
                                          cpx<T> *line, int c, int row, int t, int TPL)
{
    const bool act = (fold == 2) ? (*((volatile const int *)&st->es_mode) == 2) : (st->es_saved >= st->es_K);
    if (!act) return;
    addrP<PAD> A;
    const int K = st->es_K;
    const long long slot = (long long)3 * nrows * LX;
    const cpx<T> *g = esG + ((long long)c * nrows + row) * LX;
    for (int m = t; m < LX; m += TPL) line[A(m)] = cscale(line[A(m)], f);
#pragma unroll 1
    for (int k = 0; k < K; k++) {
        const T wk = (T)bm_es_weight(st, fold == 2, ceval, k);
        const cpx<T> *gk = g + k * slot;
        for (int m = t; m < LX; m += TPL) {
            const cpx<T> gv = gk[m];
            const cpx<T> v = line[A(m)];
            line[A(m)] = mk<T>(v.x + wk * gv.x, v.y + wk * gv.y);
        }
    }
}

// L2 prefetch of the per-cell input rows of the block whose rows start at r0 (this row and the z + 1
// row of M, the update base, the earlier stage evaluations, the material maps). Every prefetched
// address lies inside its row.
template <typename T>
__device__ __forceinline__ void stage_prefetch_rows(const StageArgs<T> &a, int r0)
{
    const int nx = a.nx, ny = a.ny, nz = a.nz, rpb = a.rpb, tid = threadIdx.x;
    const int nrows = ny * nz;
    const long long n = a.n;
    const int lpr = (int)((nx * sizeof(T) + 127) / 128);   // 128-byte lines per row
    const StageLayout L = stage_layout(a);
    const int nzr = L.ns > 1 ? 3 : 0;                        // z + 1 rows of M
    const int nev = (a.mode == BM_MODE_HEFF) ? 0 : a.nev;
    const int o_mb = 3 + nzr, o_ev = o_mb + 3 * L.mb, o_ms = o_ev + 3 * nev, o_k1 = o_ms + L.ms;
    const int nrow = o_k1 + L.k1;
    const int lsh = 32 - __clz(lpr - 1), lpr2 = 1 << lsh;   // lines per row rounded up to a power of two
    for (int job = tid; job < rpb * nrow * lpr2; job += blockDim.x) {
        const int line_i = job & (lpr2 - 1), rk = job >> lsh;
        if (line_i >= lpr) continue;
        const int r = rpb == 1 ? 0 : rk / nrow, k = rk - r * nrow;
        const int row = r0 + r;
        if (row >= nrows) continue;
        const long long ro = (long long)row * nx;
        const T *src = nullptr;
        if (k < 3) src = a.Min + k * n + ro;
        else if (k < o_mb) src = (row + ny < nrows) ? a.Min + (k - 3) * n + ro + (long long)ny * nx : nullptr;
        else if (k < o_ev) src = a.Mbase + (k - o_mb) * n + ro;
        else if (k < o_ms) src = a.ev[(k - o_ev) / 3] + ((k - o_ev) % 3) * n + ro;
        else if (k < o_k1) src = a.Ms_map + ro;
        else src = a.K1_map + ro;
        if (src) asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(src) + 128 * line_i));
    }
}

template <typename T, int LX, int XV, int SPEC = 0>
__device__ __forceinline__ void stage_reg_body(const StageArgs<T> &a, int bid, unsigned int total)
{
    extern __shared__ unsigned char smraw[];
    cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw);
    using C = xr_cfg<LX, XV>;
    constexpr int TPL = C::TPL, LSP = C::LSP;
    addrP<C::PAD> A;
    const int rpb = a.rpb;
    const int nrows = a.ny * a.nz;
    const int r0 = bid * rpb;
    const int tid = threadIdx.x;
    const int q = tid / TPL, t = tid % TPL;
    const int qc = rpb == 1 ? q : q / rpb, qr = q - qc * rpb;
    const bool qact = (q < 3 * rpb) && (r0 + qr < nrows);
    cpx<T> *line = sm + (q < 3 * rpb ? q : 0) * LSP;
    const bool demag = SPEC == 1 || SPEC == 2 || (SPEC == 0 && (a.mode != BM_MODE_UPDATE) && (a.modules & BM_MOD_DEMAG));
    const int half = (a.nx + 1) >> 1;   // packed elements that carry mesh cells
    // group 1: the spectrum rows
    if (demag && qact) {
        const cpx<T> *src = a.S1 + ((long long)qc * nrows + r0 + qr) * LX;
#pragma unroll 4
        for (int m = t; m < LX; m += TPL) cp_async_cpx<T>(&line[A(m)], &src[m], true);
    }
    cp_async_commit();
    // without staging: L2 prefetch of the rows the per-cell phase reads from DRAM, so that they arrive
    // while the inverse transform runs
    if (!a.staged && (a.mode != BM_MODE_UPDATE || a.Mbase != a.Min)) stage_prefetch_rows<T>(a, r0);
    // group 2: the per-cell input rows, arriving while the inverse transform runs
    AccStaged<T> st;
    if (a.staged) {
        const StageLayout L = stage_layout(a);
        const int nx = a.nx, ny = a.ny, nz = a.nz;
        const long long n = a.n;
        size_t lbytes = ((size_t)3 * rpb * LSP * sizeof(cpx<T>) + 15) & ~(size_t)15;
        T *R = reinterpret_cast<T *>(smraw + lbytes);
        st.R = R; st.nx = nx; st.kr = L.kr; st.ns3 = 3 * L.ns; st.hasmb = L.mb;
        st.evo = 3 * L.ns + 3 * L.mb;
        st.mso = st.evo + 3 * (a.mode == BM_MODE_HEFF ? 0 : a.nev);
        st.k1o = st.mso + L.ms;
        const bool chunk = ((nx * (int)sizeof(T)) % 16) == 0;
        const int per16 = 16 / (int)sizeof(T);
        const int CH = chunk ? nx / per16 : nx;
        const int lane = tid & 31, warp = tid >> 5, nwarp = (blockDim.x + 31) >> 5;
        const int wsz = min(32, (int)blockDim.x - warp * 32);   // lanes present in this warp
        for (int job = warp; job < rpb * L.kr; job += nwarp) {
            const int r = job / L.kr, kk = job - r * L.kr;
            const int row = r0 + r;
            if (row >= nrows) continue;
            const int y = row % ny, z = row / ny;
            const T *src = nullptr;
            if (kk < 3 * L.ns) {
                const int slot = kk / 3, c = kk - 3 * slot;
                long long srow = -1;
                if (slot == 0) srow = row;
                else if (slot == 1) srow = (y > 0) ? row - 1 : -1;
                else if (slot == 2) srow = (y + 1 < ny) ? row + 1 : -1;
                else if (slot == 3) srow = (z > 0) ? row - ny : -1;
                else srow = (z + 1 < nz) ? row + ny : -1;
                if (srow >= 0) src = a.Min + c * n + srow * nx;
            } else if (kk < st.evo) {
                src = a.Mbase + (kk - 3 * L.ns) * n + (long long)row * nx;
            } else if (kk < st.mso) {
                const int i = (kk - st.evo) / 3, c = (kk - st.evo) - 3 * i;
                src = a.ev[i] + c * n + (long long)row * nx;
            } else if (kk < st.k1o) {
                src = a.Ms_map + (long long)row * nx;
            } else {
                src = a.K1_map + (long long)row * nx;
            }
            if (!src) continue;
            T *dst = R + ((long long)r * L.kr + kk) * nx;
            if (chunk)
                for (int i = lane; i < CH; i += wsz) cp_async_el<16>(dst + i * per16, src + i * per16, true);
            else
                for (int i = lane; i < CH; i += wsz) cp_async_real<T>(dst + i, src + i, true);
        }
    }
    cp_async_commit();
    if (demag) {
        cp_async_wait_group<1>();
        __syncthreads();
        if (SPEC == 0 && a.es_fold) {
            // evaluation speedup: an extrapolating evaluation turns the row of X[M] into the
            // extrapolated field's row (the k_es_extrap sum, formed here so the spectrum is not
            // written and read back); kept out of line so the hot path's registers are untouched
            if (qact)
                es_fold_line<T, LX, C::PAD>(a.st, a.es_fold, a.esG, (T)a.es_cs[qc], a.es_ceval, nrows, line, qc, r0 + qr, t,
                                            TPL);
            __syncthreads();
        }
        if constexpr (XV == 0) xinv_pre_f<T>(line, LX, a.twx2, t, TPL, qact, A, [] { __syncthreads(); });
        else xinv_pre_f<T>(line, LX, a.twx2, t, TPL, qact, A, [] { xs_sync<TPL>(); });
        x_reg<T, LX, XV, true>(line, t, qact, a.twx, half);
    }
    cp_async_wait_group<0>();
    __syncthreads();
    double lmax = 0.0;
    if (SPEC == 0 && a.staged) stage_cells<T>(a, sm, LSP, A, r0, lmax, st);
    else stage_cells<T, SPEC>(a, sm, LSP, A, r0, lmax, AccGlobal<T>(a));
    if (SPEC == 1 || SPEC == 3 || (SPEC == 0 && a.do_xfwd)) {
        for (int idx = tid; idx < 3 * rpb * (LX / 2); idx += blockDim.x) {
            int qq = idx / (LX / 2), mm = idx - qq * (LX / 2);
            if (mm >= half) sm[qq * LSP + A(mm)] = mk<T>(0, 0);
        }
        __syncthreads();
        x_reg<T, LX, XV, false>(line, t, qact, a.twx, LX);
        // split into the packed half spectrum pairwise (k, LX - k) straight into the S1 row
        // (xfwd_post)
        if (qact) {
            cpx<T> *dst = a.S1 + ((long long)qc * nrows + r0 + qr) * LX;
            for (int k = t; k <= LX / 2; k += TPL) {
                if (k == 0) {
                    const cpx<T> z0 = line[A(0)];
                    dst[0] = mk<T>(z0.x + z0.y, z0.x - z0.y);
                    continue;
                }
                const int k2 = LX - k;
                const cpx<T> Av = line[A(k)], Bc = conj(line[A(k2)]);
                const cpx<T> E = cscale(Av + Bc, (T)0.5);
                const cpx<T> O = cscale(mul_mi(Av - Bc), (T)0.5);
                const cpx<T> wO = cmul(a.twx2[k], O);
                dst[k] = E + wO;
                if (k2 != k) dst[k2] = conj(E - wO);
            }
        }
    }
    stage_tail<T, SPEC>(a, lmax, total);
}

template <typename T, int LX>
__global__ void __launch_bounds__(bm_lb<T>::v) k_stage_reg(StageArgs<T> a)
{
    if (stage_gated_out<T>(a.st, a.gate)) return;
    stage_reg_body<T, LX, 0>(a, blockIdx.x, gridDim.x);
}

template <typename T, int LX>
__global__ void __maxnreg__(sizeof(T) == 8 ? 128 : BM_RX_MAXNREG_F) k_stage_rx(StageArgs<T> a)
{
    if (stage_gated_out<T>(a.st, a.gate)) return;
    stage_reg_body<T, LX, 1>(a, blockIdx.x, gridDim.x);
}

template <typename T, int LX, int SPEC>
__global__ void __maxnreg__(sizeof(T) == 8 ? 128 : BM_RX_MAXNREG_F) k_stage_rx16(StageArgs<T> a)
{
    if (stage_gated_out<T>(a.st, a.gate)) return;
    stage_reg_body<T, LX, 2, SPEC>(a, blockIdx.x, gridDim.x);
}

template <typename T, int LX, int SPEC>
__global__ void __maxnreg__(sizeof(T) == 8 ? 128 : BM_RX16_LO_MAXNREG_F) k_stage_rx16_lo(StageArgs<T> a)
{
    if (stage_gated_out<T>(a.st, a.gate)) return;
    stage_reg_body<T, LX, 2, SPEC>(a, blockIdx.x, gridDim.x);
}


// many meshes with the same x length in one launch (radix-8 transform): work item (mesh, row
// block); the error-norm maximum and the step bookkeeping follow k_stage_batch
template <typename T, int LX, int SPEC = 0>
__global__ void __maxnreg__(sizeof(T) == 8 ? 128 : BM_RX_MAXNREG_F) k_stage_rx_batch(const StageArgs<T> *__restrict__ args,
                                                                         const int2 *__restrict__ work, int nwork)
{
    if (stage_gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    stage_reg_body<T, LX, 1, SPEC>(args[it.x], it.y, (unsigned int)nwork);
}

template <typename T, int LX, int XV>
static int launch_stage_reg(const StageArgs<T> &a, cudaStream_t s)
{
    using C = xr_cfg<LX, XV == 3 ? 2 : XV>;
    int nt = (3 * a.rpb * C::TPL + 31) & ~31;   // whole warps: the error-norm reduction shuffles full warps
    if (nt > bm_lb<T>::v) return 203;
    size_t smem = (size_t)3 * a.rpb * C::LSP * sizeof(cpx<T>);
    if (smem > 200 * 1024) return 204;
    StageArgs<T> b = a;
    if (b.staged) {
        // stage the per-cell rows when they fit; otherwise read them from global memory
        size_t lb = (smem + 15) & ~(size_t)15;
        size_t rb = (size_t)b.rpb * stage_layout(b).kr * b.nx * sizeof(T);
        if (lb + rb <= 200 * 1024) smem = lb + rb;
        else b.staged = 0;
    }
    void (*kern)(StageArgs<T>);
    if constexpr (XV == 0) kern = k_stage_reg<T, LX>;
    else if constexpr (XV == 1) kern = k_stage_rx<T, LX>;
    else {
        const int sp = stage_plain(b) ? 1 : stage_lte_plain(b) ? 2 : stage_adv_plain(b) ? 3 : 0;
        if constexpr (XV == 2)
            kern = sp == 1 ? k_stage_rx16<T, LX, 1> : sp == 2 ? k_stage_rx16<T, LX, 2> : sp == 3 ? k_stage_rx16<T, LX, 3>
                                                                                          : k_stage_rx16<T, LX, 0>;
        else
            kern = sp == 1 ? k_stage_rx16_lo<T, LX, 1> : sp == 2 ? k_stage_rx16_lo<T, LX, 2>
                         : sp == 3 ? k_stage_rx16_lo<T, LX, 3> : k_stage_rx16_lo<T, LX, 0>;
    }
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return 2000 + (int)e;   // the shared-memory ceiling was refused
    }
    int nrows = a.ny * a.nz;
    dim3 grid((nrows + a.rpb - 1) / a.rpb);
    kern<<<grid, nt, smem, s>>>(b);
    return (int)cudaGetLastError();
}

// x lengths with a register kernel and their threads per line
int stage_reg_q(int LX, int xv)
{
    if (xv == 3) xv = 2;   // the radix-16 kernel at the lower register cap: the same shape
    switch (LX) {
    case 16: return xv == 2 ? 0 : xv ? 2 : 4;
    case 32: return xv == 2 ? 0 : xv ? 4 : 8;
    case 64: return xv == 2 ? 0 : 8;
    case 128: return xv == 2 ? 0 : 16;
    case 256: return xv == 2 ? 16 : xv ? 32 : 16;
    case 512: return xv == 2 ? 32 : xv ? 64 : 32;
    case 1024: return xv == 2 ? 64 : xv ? 128 : 32;
    case 24: case 48: case 96: case 192: case 384: case 768:
        return xv == 1 ? LX / 12 : 0;   // Stockham only
    default: return 0;
    }
}

template <typename T, int LX> static int launch_stage_xv(const StageArgs<T> &a, cudaStream_t s)
{
    if constexpr (LX >= 256) {
        // xv 3 is its own kernel for FP32 only (the FP64 cap is the same for both)
        if constexpr (sizeof(T) == 4) {
            if (a.xv == 3) return launch_stage_reg<T, LX, 3>(a, s);
        }
        if (a.xv == 2 || a.xv == 3) return launch_stage_reg<T, LX, 2>(a, s);
    }
    return a.xv ? launch_stage_reg<T, LX, 1>(a, s) : launch_stage_reg<T, LX, 0>(a, s);
}


template <typename T> int launch_stage(const StageArgs<T> &a, cudaStream_t s)
{
    switch (a.LX) {
    case 16: return launch_stage_xv<T, 16>(a, s);
    case 32: return launch_stage_xv<T, 32>(a, s);
    case 64: return launch_stage_xv<T, 64>(a, s);
    case 128: return launch_stage_xv<T, 128>(a, s);
    case 256: return launch_stage_xv<T, 256>(a, s);
    case 512: return launch_stage_xv<T, 512>(a, s);
    case 1024: return launch_stage_xv<T, 1024>(a, s);
    case 24: if (a.xv) return launch_stage_reg<T, 24, 1>(a, s); break;
    case 48: if (a.xv) return launch_stage_reg<T, 48, 1>(a, s); break;
    case 96: if (a.xv) return launch_stage_reg<T, 96, 1>(a, s); break;
    case 192: if (a.xv) return launch_stage_reg<T, 192, 1>(a, s); break;
    case 384: if (a.xv) return launch_stage_reg<T, 384, 1>(a, s); break;
    case 768: if (a.xv) return launch_stage_reg<T, 768, 1>(a, s); break;
    default: break;
    }
    int nt = (3 * a.rpb * a.px.tpl + 31) & ~31;   // whole warps
    if (nt > bm_lb<T>::v) return 201;
    size_t smem = (size_t)3 * a.rpb * padded_len(a.LX) * sizeof(cpx<T>);
    if (smem > 200 * 1024) return 202;
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_stage<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    int nrows = a.ny * a.nz;
    dim3 grid((nrows + a.rpb - 1) / a.rpb);
    k_stage<T><<<grid, nt, smem, s>>>(a);
    return (int)cudaGetLastError();
}

bool stage_reg_path(int LX, int xv)
{
    switch (LX) {
    case 16: case 32: case 64: case 128: case 256: case 512: case 1024: return true;
    case 24: case 48: case 96: case 192: case 384: case 768: return xv != 0;
    default: return false;
    }
}

template int launch_stage<float>(const StageArgs<float> &, cudaStream_t);
template int launch_stage<double>(const StageArgs<double> &, cudaStream_t);

// radix-16 variant (x lengths 256 .. 1024)
template <typename T, int LX, int SPEC = 0>
__global__ void __maxnreg__(sizeof(T) == 8 ? 128 : BM_RX_MAXNREG_F) k_stage_rx16_batch(const StageArgs<T> *__restrict__ args,
                                                                                       const int2 *__restrict__ work, int nwork)
{
    if (stage_gated_out<T>(args[0].st, args[0].gate) || (int)blockIdx.x >= nwork) return;
    const int2 it = work[blockIdx.x];
    stage_reg_body<T, LX, 2, SPEC>(args[it.x], it.y, (unsigned int)nwork);
}

template <typename T, int LX, int SPEC>
static int launch_stage_rx_batch_s(const StageArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s)
{
    if constexpr (LX >= 256 && (LX % 3) != 0) {
        if (smem > BM_SMEM_DEFAULT_SAFE) {
            cudaError_t e = cudaFuncSetAttribute(k_stage_rx16_batch<T, LX, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 BM_SMEM_CAP);
            if (e != cudaSuccess) return 2000 + (int)e;
        }
        k_stage_rx16_batch<T, LX, SPEC><<<nwork, nt, smem, s>>>(dargs, dwork, nwork);
        return (int)cudaGetLastError();
    }
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_stage_rx_batch<T, LX, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    k_stage_rx_batch<T, LX, SPEC><<<nwork, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

// the plain-stage instantiation for FP32 launches whose argument blocks are all plain (stage_plain)
template <typename T, int LX>
static int launch_stage_rx_batch(const StageArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s,
                                 int plain)
{
    if constexpr (sizeof(T) == 4) {
        if (plain) return launch_stage_rx_batch_s<T, LX, 1>(dargs, dwork, nwork, nt, smem, s);
    }
    return launch_stage_rx_batch_s<T, LX, 0>(dargs, dwork, nwork, nt, smem, s);
}

template <typename T>
int launch_stage_batch(int key, const StageArgs<T> *dargs, const int2 *dwork, int nwork, int nt, size_t smem, cudaStream_t s,
                       int plain)
{
    if (nwork < 1) return 0;
    if (nt > bm_lb<T>::v || nt < 32) return 211;
    if (smem > 200 * 1024) return 212;
    switch (key) {
    case 0: break;
    case 16: return launch_stage_rx_batch<T, 16>(dargs, dwork, nwork, nt, smem, s, plain);
    case 32: return launch_stage_rx_batch<T, 32>(dargs, dwork, nwork, nt, smem, s, plain);
    case 64: return launch_stage_rx_batch<T, 64>(dargs, dwork, nwork, nt, smem, s, plain);
    case 128: return launch_stage_rx_batch<T, 128>(dargs, dwork, nwork, nt, smem, s, plain);
    case 256: return launch_stage_rx_batch<T, 256>(dargs, dwork, nwork, nt, smem, s, plain);
    case 512: return launch_stage_rx_batch<T, 512>(dargs, dwork, nwork, nt, smem, s, plain);
    case 1024: return launch_stage_rx_batch<T, 1024>(dargs, dwork, nwork, nt, smem, s, plain);
    case 24: return launch_stage_rx_batch<T, 24>(dargs, dwork, nwork, nt, smem, s, plain);
    case 48: return launch_stage_rx_batch<T, 48>(dargs, dwork, nwork, nt, smem, s, plain);
    case 96: return launch_stage_rx_batch<T, 96>(dargs, dwork, nwork, nt, smem, s, plain);
    case 192: return launch_stage_rx_batch<T, 192>(dargs, dwork, nwork, nt, smem, s, plain);
    case 384: return launch_stage_rx_batch<T, 384>(dargs, dwork, nwork, nt, smem, s, plain);
    case 768: return launch_stage_rx_batch<T, 768>(dargs, dwork, nwork, nt, smem, s, plain);
    default: return 213;
    }
    if (smem > BM_SMEM_DEFAULT_SAFE) {
        cudaError_t e = cudaFuncSetAttribute(k_stage_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, BM_SMEM_CAP);
        if (e != cudaSuccess) return (int)e;
    }
    k_stage_batch<T><<<nwork, nt, smem, s>>>(dargs, dwork, nwork);
    return (int)cudaGetLastError();
}

template int launch_stage_batch<float>(int, const StageArgs<float> *, const int2 *, int, int, size_t, cudaStream_t, int);
template int launch_stage_batch<double>(int, const StageArgs<double> *, const int2 *, int, int, size_t, cudaStream_t, int);
