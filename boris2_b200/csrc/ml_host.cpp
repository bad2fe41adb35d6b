// Host geometry of the multilayered convolution.
//
// Follows the reference's rules so that the same meshes give the same layers, common grid,
// transfer weights and kernel collection:
//   n_common         SDemag::set_default_n_common (Boris/SDemag.cpp:173), Set_n_common (:362),
//                    Set_2D_Multilayered_Convolution (:341)
//   layer rectangles SDemag::set_Rect_collection (Boris/SDemag.cpp:215); 2D-layered mode takes
//                    Rect::get_zlayer of every z cell layer (BorisLib/Types_Rect.h:485)
//   h_max            SDemag::get_maximum_cellsize (Boris/SDemag.cpp:297), over the meshes' own h
//   transfer flag    SDemag_Demag::Initialize (Boris/SDemag_Demag.cpp:349)
//   transfer weights MESHTRANSFERTYPE_WEIGHTED in BorisLib/VEC_MeshTransfer.h: in direction
//                    :901 (covered-volume ratio times reciprocal-distance weights, :306), out
//                    direction :1221 (reciprocal-distance weights, :396); floor/ceil with the
//                    1e-4 rounding margin (BorisLib/Funcs_Math.h:161) and 1e-12 comparisons
//                    (BorisLib/Funcs_Aux_base.h:9)
//   kernel reuse     DemagKernelCollection::Calculate_Demag_Kernels / KernelAlreadyComputed
//                    (Boris/DemagKernelCollection_Calc.cpp:9,114): one kernel per (shift,
//                    h_src, h_dst); in 2D a kernel of the opposite z shift is reused with the
//                    xz, yz signs flipped
//   kernel kinds     KerType::AllocateKernels (Boris/DemagKernelCollection.cpp:8): self, z-shifted
//                    or full complex
#include "ml.h"
#include <cmath>
#include <algorithm>

namespace {

const double kEps = 1e-12;
const double kRound = 1e-4;

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() {}
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    V3 operator+(const V3 &o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3 &o) const { return V3(x - o.x, y - o.y, z - o.z); }
    double norm() const { return std::sqrt(x * x + y * y + z * z); }
    double &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct Box {
    V3 s, e;
    V3 size() const { return e - s; }
};

bool zero(double v) { return v < kEps && v > -kEps; }
bool zero_or_pos(double v) { return v > 0 || zero(v); }
bool same(const V3 &a, const V3 &b) { return zero(a.x - b.x) && zero(a.y - b.y) && zero(a.z - b.z); }
bool same(const Box &a, const Box &b) { return same(a.s, b.s) && same(a.e, b.e); }
double floor_r(double v) { return std::floor(v + kRound); }
double ceil_r(double v) { return std::ceil(v - kRound); }

// intersection with the reference's closed-interval test; false when it is the null box
bool intersection(const Box &a, const Box &b, Box &r)
{
    V3 st(std::max(a.s.x, b.s.x), std::max(a.s.y, b.s.y), std::max(a.s.z, b.s.z));
    V3 en(std::min(a.e.x, b.e.x), std::min(a.e.y, b.e.y), std::min(a.e.z, b.e.z));
    r = Box();
    if (zero_or_pos(en.x - st.x) && zero_or_pos(en.y - st.y) && zero_or_pos(en.z - st.z)) { r.s = st; r.e = en; }
    return !(zero(r.s.x) && zero(r.s.y) && zero(r.s.z) && zero(r.e.x) && zero(r.e.y) && zero(r.e.z));
}
bool is_plane(const Box &r)
{
    double dx = r.s.x - r.e.x, dy = r.s.y - r.e.y, dz = r.s.z - r.e.z;
    return (zero(dx) && !zero(dy) && !zero(dz)) || (zero(dy) && !zero(dx) && !zero(dz)) || (zero(dz) && !zero(dx) && !zero(dy));
}
bool is_point(const Box &r) { return same(r.s, r.e); }

// cells of a grid (n, h, origin) inside the floor/ceil index box of rc, with reciprocal
// distance weights (d_max - distance to the centre of rc); returns their sum
double recip_weights(const Box &rc, const int n[3], const V3 &h, const V3 &origin, std::vector<int> &idx,
                     std::vector<double> &w)
{
    V3 coord = V3((rc.e.x + rc.s.x) / 2, (rc.e.y + rc.s.y) / 2, (rc.e.z + rc.s.z) / 2) - origin;
    V3 pll = rc.s - origin, pur = rc.e - origin;
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        lo[a] = (int)floor_r(pll[a] / h[a]);
        hi[a] = (int)ceil_r(pur[a] / h[a]);
        lo[a] = std::max(lo[a], 0);
        hi[a] = std::min(hi[a], n[a]);
    }
    V3 sz = rc.size();
    double dmax = V3(sz.x / 2 + h.x / 2, sz.y / 2 + h.y / 2, sz.z / 2 + h.z / 2).norm();
    double tot = 0.0;
    for (int i = lo[0]; i < hi[0]; i++)
        for (int j = lo[1]; j < hi[1]; j++)
            for (int k = lo[2]; k < hi[2]; k++) {
                V3 cc((i + 0.5) * h.x, (j + 0.5) * h.y, (k + 0.5) * h.z);
                double dr = dmax - (cc - coord).norm();
                tot += dr;
                idx.push_back(i + j * n[0] + k * n[0] * n[1]);
                w.push_back(dr);
            }
    return tot;
}

int nice(int n)
{
    int best = 1;
    while (best < n) best *= 2;
    for (int t = 3; t < best; t *= 2)
        if (t >= n) { best = t; break; }
    return best;
}

}  // namespace

int ml_build_geometry(const std::vector<MLMeshIn> &meshes, int mode, const int *nc_user, MLGeom &g, std::string &err)
{
    g = MLGeom();
    const int nm = (int)meshes.size();
    if (nm < 1) { err = "multilayer: no mesh with demag"; return 1; }
    std::vector<Box> mrect(nm);
    std::vector<V3> mh(nm);
    for (int m = 0; m < nm; m++) {
        mh[m] = V3(meshes[m].h[0], meshes[m].h[1], meshes[m].h[2]);
        mrect[m].s = V3(meshes[m].o[0], meshes[m].o[1], meshes[m].o[2]);
        mrect[m].e = mrect[m].s + V3(mh[m].x * meshes[m].n[0], mh[m].y * meshes[m].n[1], mh[m].z * meshes[m].n[2]);
    }
    // n_common and the 2D mode
    int force2d = mode;
    if (nc_user) {
        for (int a = 0; a < 3; a++) g.nc[a] = nc_user[a];
        if (force2d == 0 && g.nc[2] == 1) force2d = 1;
    } else {
        bool all2d = true;
        for (int m = 0; m < nm; m++) {
            if (meshes[m].n[2] != 1) all2d = false;
            for (int a = 0; a < 3; a++) g.nc[a] = std::max(g.nc[a], meshes[m].n[a]);
        }
        if (all2d) g.nc[2] = 1;
    }
    if (force2d) g.nc[2] = 1;
    for (int a = 0; a < 3; a++)
        if (g.nc[a] < 1) { err = "multilayer: n_common must be >= 1"; return 1; }
    g.force2d = force2d;
    for (int a = 0; a < 3; a++) g.N[a] = (a < 2 || g.nc[2] > 1) ? 2 * nice(g.nc[a]) : 1;
    // layers and their raw rectangles
    std::vector<Box> rc;
    for (int m = 0; m < nm; m++) {
        int nl = (force2d == 2) ? meshes[m].n[2] : 1;
        for (int q = 0; q < nl; q++) {
            Box r = mrect[m];
            if (force2d == 2) {
                double t = mh[m].z;
                if (!(q * t < 0 || (q + 1) * t > (r.e.z - r.s.z))) {
                    r.s.z = mrect[m].s.z + q * t;
                    r.e.z = mrect[m].s.z + (q + 1) * t;
                }
            }
            MLLayerGeom L;
            L.mesh = m;
            L.zlayer = (force2d == 2) ? q : -1;
            g.layers.push_back(L);
            rc.push_back(r);
        }
    }
    g.L = (int)rc.size();
    if (g.L > BM_ML_MAXL) { err = "multilayer: more than " + std::to_string(BM_ML_MAXL) + " layers"; return 1; }
    // enlarge every rectangle to the largest size, starting as close as possible to the smallest start
    V3 mx;
    V3 mn = rc[0].s;
    for (auto &r : rc) {
        V3 sz = r.size();
        for (int a = 0; a < 3; a++) {
            if (mx[a] < sz[a]) mx[a] = sz[a];
            if (r.s[a] < mn[a]) mn[a] = r.s[a];
        }
    }
    for (auto &r : rc)
        for (int a = 0; a < 3; a++) {
            if (a == 2 && g.nc[2] == 1) continue;   // 2D: layers keep their thickness
            if (r.e[a] - mx[a] < mn[a]) { r.s[a] = mn[a]; r.e[a] = r.s[a] + mx[a]; }
            else r.s[a] = r.e[a] - mx[a];
        }
    for (int l = 0; l < g.L; l++) {
        MLLayerGeom &y = g.layers[l];
        V3 sz = rc[l].size();
        for (int a = 0; a < 3; a++) { y.rs[a] = rc[l].s[a]; y.re[a] = rc[l].e[a]; y.hc[a] = sz[a] / g.nc[a]; }
        double hm = std::max(mh[y.mesh].x, std::max(mh[y.mesh].y, mh[y.mesh].z));
        g.h_max = std::max(g.h_max, hm);
    }
    // kernel collection
    struct KD { V3 shift, hs, hd; };
    std::vector<KD> kd;
    g.pair_kernel.assign(g.L * g.L, -1);
    g.pair_inv.assign(g.L * g.L, 0);
    g.pair_kind.assign(g.L * g.L, 0);
    const bool two_d = (g.nc[2] == 1);
    const double hmx = g.h_max;
    for (int d = 0; d < g.L; d++) {
        V3 hdst(g.layers[d].hc[0], g.layers[d].hc[1], g.layers[d].hc[2]);
        for (int s = 0; s < g.L; s++) {
            V3 shift = rc[d].s - rc[s].s;
            V3 hsrc(g.layers[s].hc[0], g.layers[s].hc[1], g.layers[s].hc[2]);
            int found = -1;
            // search the collections in order, each over its kernels in source order
            for (int c2 = 0; c2 < g.L && found < 0; c2++)
                for (int k2 = 0; k2 < g.L && found < 0; k2++) {
                    int kk = g.pair_kernel[c2 * g.L + k2];
                    if (kk < 0) continue;
                    if (!(same(kd[kk].hs, hsrc) && same(kd[kk].hd, hdst))) continue;
                    if (same(kd[kk].shift, shift)) found = kk;
                    else if (two_d && zero(shift.x) && zero(shift.y) && zero(kd[kk].shift.x) && zero(kd[kk].shift.y) &&
                             zero(shift.z + kd[kk].shift.z))
                        found = kk;
                }
            const bool self = same(rc[s], rc[d]);
            int inv = 0;
            if (found >= 0) {
                if (zero(shift.x) && zero(shift.y) && !zero(shift.z) && zero(shift.z + kd[found].shift.z)) inv = 1;
            } else {
                MLKernelSpec K;
                KD k;
                if (self) {
                    k.shift = V3(); k.hs = hdst; k.hd = hdst;
                    K.kind = BM_MLK_SELF;
                    K.irregular = 0;
                    for (int a = 0; a < 3; a++) { K.hs[a] = K.hd[a] = hdst[a] / hmx; K.shift[a] = 0.0; }
                } else {
                    k.shift = shift; k.hs = hsrc; k.hd = hdst;
                    K.kind = (zero(shift.x) && zero(shift.y)) ? BM_MLK_ZSHIFT : BM_MLK_FULL;
                    for (int a = 0; a < 3; a++) K.shift[a] = shift[a] / hmx;
                    if (two_d) {
                        for (int a = 0; a < 3; a++) { K.hs[a] = hsrc[a] / hmx; K.hd[a] = hdst[a] / hmx; }
                        // irregular unless s * 1e-9 == d * 1e-9 (Boris/DemagTFunc_Irregular.cpp:12)
                        K.irregular = same(V3(K.hs[0] * 1e-9, K.hs[1] * 1e-9, K.hs[2] * 1e-9),
                                           V3(K.hd[0] * 1e-9, K.hd[1] * 1e-9, K.hd[2] * 1e-9)) ? 0 : 1;
                    } else {
                        // 3D uses the destination cellsize throughout (Boris/DemagKernelCollection_Calc.cpp:921)
                        K.irregular = 0;
                        for (int a = 0; a < 3; a++) K.hs[a] = K.hd[a] = hdst[a] / hmx;
                    }
                }
                found = (int)kd.size();
                kd.push_back(k);
                g.kernels.push_back(K);
            }
            g.pair_kernel[d * g.L + s] = found;
            g.pair_inv[d * g.L + s] = inv;
            if (self) g.pair_kind[d * g.L + s] = 1;
            else if (g.kernels[found].kind == BM_MLK_ZSHIFT) g.pair_kind[d * g.L + s] = inv ? 3 : 2;
            else g.pair_kind[d * g.L + s] = (g.kernels[found].kind == BM_MLK_SELF) ? 1 : 4;
        }
    }
    // transfers
    const int ncc = g.nc[0] * g.nc[1] * g.nc[2];
    g.out.assign(nm, MLMeshOut());
    std::vector<std::vector<std::vector<int>>> oidx(nm);
    std::vector<std::vector<std::vector<double>>> ow(nm);
    for (int l = 0; l < g.L; l++) {
        MLLayerGeom &y = g.layers[l];
        const int m = y.mesh;
        V3 hc(y.hc[0], y.hc[1], y.hc[2]);
        y.transfer = !(same(rc[l], mrect[m]) && same(hc, mh[m]));
        if (!y.transfer) continue;
        y.in_ptr.assign(ncc + 1, 0);
        for (int c = 0; c < ncc; c++) {
            int i = c % g.nc[0], j = (c / g.nc[0]) % g.nc[1], k = c / (g.nc[0] * g.nc[1]);
            Box cell;
            cell.s = rc[l].s + V3(hc.x * i, hc.y * j, hc.z * k);
            cell.e = cell.s + hc;
            Box ri;
            std::vector<int> idx;
            std::vector<double> w;
            double tot = 0.0, cov = 0.0;
            if (intersection(mrect[m], cell, ri) && !is_plane(ri) && !is_point(ri)) {
                V3 si = ri.size(), sc = cell.size();
                cov += (si.x / sc.x) * (si.y / sc.y) * (si.z / sc.z);
                tot += recip_weights(cell, meshes[m].n, mh[m], mrect[m].s, idx, w);
            }
            if (tot > 0)
                for (auto &v : w) v *= cov / tot;
            y.in_idx.insert(y.in_idx.end(), idx.begin(), idx.end());
            y.in_w.insert(y.in_w.end(), w.begin(), w.end());
            y.in_ptr[c + 1] = (int)y.in_idx.size();
        }
        // out direction, into this mesh's block list
        const int n = meshes[m].n[0] * meshes[m].n[1] * meshes[m].n[2];
        const int block = (int)g.out[m].layers.size();
        g.out[m].layers.push_back(l);
        if (oidx[m].empty()) { oidx[m].resize(n); ow[m].resize(n); }
        for (int c = 0; c < n; c++) {
            int i = c % meshes[m].n[0], j = (c / meshes[m].n[0]) % meshes[m].n[1], k = c / (meshes[m].n[0] * meshes[m].n[1]);
            Box cell;
            cell.s = mrect[m].s + V3(mh[m].x * i, mh[m].y * j, mh[m].z * k);
            cell.e = cell.s + mh[m];
            std::vector<int> idx;
            std::vector<double> w;
            double tot = recip_weights(cell, g.nc, hc, rc[l].s, idx, w);
            for (size_t q = 0; q < idx.size(); q++) {
                oidx[m][c].push_back(block * 3 * ncc + idx[q]);
                ow[m][c].push_back(tot > 0 ? w[q] * (1.0 / tot) : w[q]);
            }
        }
    }
    for (int m = 0; m < nm; m++) {
        if (oidx[m].empty()) continue;
        MLMeshOut &o = g.out[m];
        const int n = (int)oidx[m].size();
        o.ptr.assign(n + 1, 0);
        for (int c = 0; c < n; c++) {
            o.idx.insert(o.idx.end(), oidx[m][c].begin(), oidx[m][c].end());
            o.w.insert(o.w.end(), ow[m][c].begin(), ow[m][c].end());
            o.ptr[c + 1] = (int)o.idx.size();
        }
    }
    // device storage of the kernels (elements of the compute type)
    const size_t Kx1 = g.N[0] / 2 + 1, Ky1 = g.N[1] / 2 + 1, Kz1 = g.N[2] / 2 + 1;
    size_t off = 0;
    for (auto &K : g.kernels) {
        if (K.kind == BM_MLK_SELF) K.count = 6 * Kx1 * Ky1 * Kz1;
        else if (K.kind == BM_MLK_ZSHIFT) K.count = 2 * 6 * Kx1 * Ky1 * Kz1;
        else K.count = 2 * 6 * Kx1 * (size_t)g.N[1] * g.N[2];
        K.off = off;
        off += (K.count + 31) & ~(size_t)31;
    }
    return 0;
}

// ------------------------------------------------------------------------------ supermesh
int sm_build_geometry(const std::vector<MLMeshIn> &meshes, const double h_request[3], SMGeom &g, std::string &err)
{
    g = SMGeom();
    const int nm = (int)meshes.size();
    if (nm < 1) { err = "supermesh: no mesh with demag"; return 1; }
    for (int a = 0; a < 3; a++)
        if (!(h_request[a] > 0)) { err = "supermesh: cellsize must be > 0"; return 1; }
    std::vector<Box> mrect(nm);
    std::vector<V3> mh(nm);
    Box u;
    bool first = true;
    for (int m = 0; m < nm; m++) {
        mh[m] = V3(meshes[m].h[0], meshes[m].h[1], meshes[m].h[2]);
        mrect[m].s = V3(meshes[m].o[0], meshes[m].o[1], meshes[m].o[2]);
        mrect[m].e = mrect[m].s + V3(mh[m].x * meshes[m].n[0], mh[m].y * meshes[m].n[1], mh[m].z * meshes[m].n[2]);
        if (first) { u = mrect[m]; first = false; continue; }
        for (int a = 0; a < 3; a++) {
            u.s[a] = std::min(u.s[a], mrect[m].s[a]);
            u.e[a] = std::max(u.e[a], mrect[m].e[a]);
        }
    }
    V3 sz = u.size();
    V3 hs;
    for (int a = 0; a < 3; a++) {
        long long c = std::llround(sz[a] / h_request[a]);
        if (c < 1) c = 1;
        if (c > (1 << 20)) { err = "supermesh: more than 2^20 cells along an axis"; return 1; }
        g.n[a] = (int)c;
        hs[a] = sz[a] / g.n[a];
        g.h[a] = hs[a];
        g.rs[a] = u.s[a];
        g.re[a] = u.e[a];
    }
    const long long ncell = (long long)g.n[0] * g.n[1] * g.n[2];
    g.mesh.assign(nm, SMMeshXfer());
    for (int m = 0; m < nm; m++) g.mesh[m].in_ptr.assign(ncell + 1, 0);
    // in: every supermesh cell gathers from every mesh it overlaps; one normalisation over all of them
    std::vector<std::vector<int>> idx(nm);
    std::vector<std::vector<double>> w(nm);
    for (long long c = 0; c < ncell; c++) {
        int i = (int)(c % g.n[0]), j = (int)((c / g.n[0]) % g.n[1]), k = (int)(c / ((long long)g.n[0] * g.n[1]));
        Box cell;
        cell.s = u.s + V3(hs.x * i, hs.y * j, hs.z * k);
        cell.e = cell.s + hs;
        double tot = 0.0, cov = 0.0;
        std::vector<size_t> start(nm);
        for (int m = 0; m < nm; m++) start[m] = idx[m].size();
        for (int m = 0; m < nm; m++) {
            Box ri;
            if (intersection(mrect[m], cell, ri) && !is_plane(ri) && !is_point(ri)) {
                V3 si = ri.size(), sc = cell.size();
                cov += (si.x / sc.x) * (si.y / sc.y) * (si.z / sc.z);
                tot += recip_weights(cell, meshes[m].n, mh[m], mrect[m].s, idx[m], w[m]);
            }
        }
        if (cov > 0) g.nonempty++;
        for (int m = 0; m < nm; m++) {
            if (tot > 0)
                for (size_t q = start[m]; q < w[m].size(); q++) w[m][q] *= cov / tot;
            g.mesh[m].in_ptr[c + 1] = (int)idx[m].size();
        }
    }
    for (int m = 0; m < nm; m++) { g.mesh[m].in_idx = idx[m]; g.mesh[m].in_w = w[m]; }
    // out: every mesh cell gathers from the supermesh cells it overlaps
    for (int m = 0; m < nm; m++) {
        SMMeshXfer &x = g.mesh[m];
        const int n = meshes[m].n[0] * meshes[m].n[1] * meshes[m].n[2];
        x.out_ptr.assign(n + 1, 0);
        for (int c = 0; c < n; c++) {
            int i = c % meshes[m].n[0], j = (c / meshes[m].n[0]) % meshes[m].n[1], k = c / (meshes[m].n[0] * meshes[m].n[1]);
            Box cell;
            cell.s = mrect[m].s + V3(mh[m].x * i, mh[m].y * j, mh[m].z * k);
            cell.e = cell.s + mh[m];
            std::vector<int> oi;
            std::vector<double> ow;
            double tot = recip_weights(cell, g.n, hs, u.s, oi, ow);
            for (size_t q = 0; q < oi.size(); q++) {
                x.out_idx.push_back(oi[q]);
                x.out_w.push_back(tot > 0 ? ow[q] * (1.0 / tot) : ow[q]);
            }
            x.out_ptr[c + 1] = (int)x.out_idx.size();
        }
    }
    return 0;
}
