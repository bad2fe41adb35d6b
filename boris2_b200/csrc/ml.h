// Multilayered demag convolution (the reference's SDemag multilayer mode): several meshes, or
// the z cell layers of meshes, convolved on one common grid with an L x L set of kernels.
//
// Host side (ml_host.cpp): layer geometry, the weighted mesh transfer to and from the common
// grid, and the kernel collection with its de-duplication. Device side (ml.cu, tensor.cu):
// transfer gathers, the fused z pass with the L x L product, and the shifted kernel build.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include <vector>
#include <string>

#define BM_ML_MAXL 8   // layers in one multilayered convolution

// kernel storage kinds on the device
#define BM_MLK_SELF 0    // real, symmetric in x, y, z: 6 planes of (Nx/2+1)(Ny/2+1)(Nz/2+1)
#define BM_MLK_ZSHIFT 1  // complex, x/y parity, Hermitian in z: 6 planes of (Nx/2+1)(Ny/2+1)(Nz/2+1)
#define BM_MLK_FULL 2    // complex, no symmetry used: 6 planes of (Nx/2+1) Ny Nz

// one mesh as the multilayer geometry sees it
struct MLMeshIn {
    int n[3];
    double h[3], o[3];
};

// one unique kernel of the collection
struct MLKernelSpec {
    int kind;            // BM_MLK_*
    int irregular;       // 2D with source and destination thickness differing
    double hs[3], hd[3]; // source / destination cellsize, normalised by h_max
    double shift[3];     // destination minus source rectangle start, normalised by h_max
    size_t off;          // offset of the kernel in the device buffer (elements of T)
    size_t count;        // elements of T
};

struct MLLayerGeom {
    int mesh;            // index into the MLMeshIn list
    int zlayer;          // z cell layer (2D-layered mode), -1 for the whole mesh
    double rs[3], re[3]; // convolution rectangle
    double hc[3];        // common-grid cellsize (rectangle / n_common)
    int transfer;        // 0: the mesh grid is the common grid (no transfer)
    // transfer in: per common cell, (mesh cell, weight)
    std::vector<int> in_ptr, in_idx;
    std::vector<double> in_w;
};

// transfer out of one mesh: per mesh cell, (layer-block element, weight) over the common-grid
// fields of the mesh's layers stored one after another ([layer][component][cell] blocks)
struct MLMeshOut {
    std::vector<int> ptr, idx;
    std::vector<double> w;
    std::vector<int> layers;   // the mesh's layers in block order
};

struct MLGeom {
    int L = 0;
    int nc[3] = {1, 1, 1};
    int N[3] = {1, 1, 1};
    int force2d = 0;
    double h_max = 0.0;
    std::vector<MLLayerGeom> layers;
    std::vector<MLKernelSpec> kernels;
    std::vector<int> pair_kernel;   // [dest * L + src]
    std::vector<int> pair_inv;      // opposite z shift reused with the xz, yz signs flipped
    std::vector<int> pair_kind;     // 1 self, 2 z-shifted, 3 inverse z-shifted, 4 full (reference naming)
    std::vector<MLMeshOut> out;     // per mesh (empty for meshes without transfer)
};

// Builds the geometry; mode 0: 3D (2D when every mesh is one cell thick or nc_user[2] == 1),
// 1: 2D, 2: 2D with every z cell layer its own layer. nc_user may be null (default n_common).
// N is the project's FFT size 2 * nice(n_common) per axis. Returns 0 or sets err.
int ml_build_geometry(const std::vector<MLMeshIn> &meshes, int mode, const int *nc_user, MLGeom &g, std::string &err);

// ------------------------------------------------------------------------------ supermesh
// Supermesh demag (the reference's SDemag with the multilayered convolution off, Boris/SDemag.cpp:
// 737-760): one convolution on the grid that spans every magnetic mesh, the meshes' M moved onto it
// and the field moved back by the weighted mesh transfer.
struct SMMeshXfer {
    // in: per supermesh cell, (cell of this mesh, weight); weights already carry the normalisation
    // over every mesh that covers the supermesh cell
    std::vector<int> in_ptr, in_idx;
    std::vector<double> in_w;
    // out: per cell of this mesh, (supermesh cell, weight)
    std::vector<int> out_ptr, out_idx;
    std::vector<double> out_w;
};

struct SMGeom {
    int n[3] = {1, 1, 1};           // supermesh cells
    double h[3] = {0, 0, 0};        // supermesh cellsize (the requested one adjusted to divide the rectangle)
    double rs[3] = {0, 0, 0}, re[3] = {0, 0, 0};   // supermesh rectangle
    long long nonempty = 0;         // supermesh cells covered by a mesh
    std::vector<SMMeshXfer> mesh;   // per input mesh
};

// Supermesh rectangle: the bounding box of the meshes (Rect::operator+=, BorisLib/Types_Rect.h:290);
// cells: round(size / h_request) per axis, at least 1, and h = size / cells
// (SuperMesh::UpdateConfiguration, Boris/SuperMeshControl.cpp:22-44); transfer weights of
// MESHTRANSFERTYPE_WEIGHTED over several input meshes (BorisLib/VEC_MeshTransfer.h:901,1221).
int sm_build_geometry(const std::vector<MLMeshIn> &meshes, const double h_request[3], SMGeom &g, std::string &err);

// ------------------------------------------------------------------------------ device arguments
// one unique kernel as the z pass sees it: storage kind, element offset in the kernel buffer,
// byte offset of its staged tile in shared memory
struct MLUDesc {
    int kind, sm;
    long long off;
};

template <typename T>
struct MLZArgs {
    cpx<T> *S2[BM_ML_MAXL];   // per layer [3][nz][Ny][LX]
    const T *K;               // kernel buffer
    MLUDesc u[BM_ML_MAXL * BM_ML_MAXL];
    unsigned char pu[BM_ML_MAXL * BM_ML_MAXL];     // (dest, src) -> unique kernel
    unsigned char pinv[BM_ML_MAXL * BM_ML_MAXL];   // (dest, src) reuses the opposite z shift
    const cpx<T> *twz;
    int L, nu, nz, Ny, Nz, LX, W;
    int ksm;                  // bytes of staged kernel tiles
    StepState *st;
    int gate;
};

// bytes of one unique kernel's staged tile at a block's columns (16-aligned):
//   self     [comp][kz <= Nz/2][W] real and the Nyquist column [comp][kz <= Nz/2] real
//   z-shift  [comp][kz <= Nz/2][W] complex and the Nyquist column [comp][kz <= Nz/2] complex
//   full     [comp][kz][pencil][W] complex and the Nyquist column [comp][kz][pencil] complex
template <typename T> BM_HD int zmid_ml_tile_main(int kind, int Nz, int W)
{
    size_t b = (kind == BM_MLK_FULL) ? (size_t)12 * Nz * W * sizeof(cpx<T>)
             : (kind == BM_MLK_SELF) ? (size_t)6 * (Nz / 2 + 1) * W * sizeof(T)
                                     : (size_t)6 * (Nz / 2 + 1) * W * sizeof(cpx<T>);
    return (int)((b + 15) & ~(size_t)15);
}
template <typename T> BM_HD int zmid_ml_tile_bytes(int kind, int Nz, int W)
{
    size_t nyq = (kind == BM_MLK_FULL) ? (size_t)12 * Nz * sizeof(cpx<T>)
               : (kind == BM_MLK_SELF) ? (size_t)6 * (Nz / 2 + 1) * sizeof(T)
                                       : (size_t)6 * (Nz / 2 + 1) * sizeof(cpx<T>);
    return zmid_ml_tile_main<T>(kind, Nz, W) + (int)((nyq + 15) & ~(size_t)15);
}
template <typename T> size_t zmid_ml_smem(int L, int Nz, int W, int ksm)
{
    // In, the kernel tiles, and the column-0 results [L][3][2][Nz]
    return (size_t)L * 3 * 2 * Nz * W * sizeof(cpx<T>) + (size_t)ksm + (size_t)L * 6 * Nz * sizeof(cpx<T>);
}
template <typename T> int launch_zmid_ml(const MLZArgs<T> &a, cudaStream_t s);
bool zmid_ml_supported(int Nz);

// dst[c * dst_plane + i] = sum_q w[q] * src[idx[q] + c * src_plane], q in [ptr[i], ptr[i+1])
// (add != 0: dst += instead of dst =)
template <typename T>
int launch_ml_gather(T *dst, long long n_dst, long long dst_plane, const T *src, long long src_plane, const int *ptr,
                     const int *idx, const T *w, StepState *st, int gate, cudaStream_t s, int add = 0);

// kernel build: 6 components of one shifted kernel (type T) into K (layout by kind)
template <typename T>
int build_ml_kernel_device(T *K, const MLKernelSpec &spec, const int *nc, const int *N, const double *farq_dev,
                           const cpx<double> *twx, const cpx<double> *twy, const cpx<double> *twz, cudaStream_t s);
