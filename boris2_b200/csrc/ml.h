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

// ------------------------------------------------------------------------------ device arguments
struct MLKDesc {
    int kind, inv;
    long long off;
};

template <typename T>
struct MLZArgs {
    cpx<T> *S2[BM_ML_MAXL];   // per layer [3][nz][Ny][LX]
    const T *K;               // kernel buffer
    MLKDesc kd[BM_ML_MAXL * BM_ML_MAXL];
    const cpx<T> *twz;
    int L, nz, Ny, Nz, LX, W;
    StepState *st;
    int gate;
};

template <typename T> int launch_zmid_ml(const MLZArgs<T> &a, cudaStream_t s);
template <typename T> size_t zmid_ml_smem(int L, int Nz, int W) { return (size_t)2 * L * 3 * 2 * Nz * W * sizeof(cpx<T>); }
bool zmid_ml_supported(int Nz);

// dst[c * dst_plane + i] = sum_q w[q] * src[idx[q] + c * src_plane], q in [ptr[i], ptr[i+1])
template <typename T>
int launch_ml_gather(T *dst, long long n_dst, long long dst_plane, const T *src, long long src_plane, const int *ptr,
                     const int *idx, const T *w, StepState *st, int gate, cudaStream_t s);

// kernel build: 6 components of one shifted kernel (type T) into K (layout by kind)
template <typename T>
int build_ml_kernel_device(T *K, const MLKernelSpec &spec, const int *nc, const int *N, const double *farq_dev,
                           const cpx<double> *twx, const cpx<double> *twy, const cpx<double> *twz, cudaStream_t s);
