// sil_internal.cuh -- shared definitions of the sm_100a DEC library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/sil_b200.h"

namespace sil {

constexpr int kMaxDims = SIL_MAX_DIMS;
constexpr int kMaxN = 4;       // form dimensions handled by d / d^T
constexpr int kMaxNHodge = 3;  // form dimensions handled by the Hodge-star based operators
constexpr int kMaxComp = 6;    // C(4,2)
constexpr int kMaxFaces = 8;   // 2 (k+1) for k+1 <= 4

// ---------------------------------------------------------------- errors

void set_error(std::string const& msg);
sil_status fail(sil_status status, std::string const& msg);
sil_status cuda_fail(cudaError_t err, char const* what);

#define SIL_CUDA_CHECK(call)                                 \
    do {                                                     \
        cudaError_t const err_ = (call);                     \
        if (err_ != cudaSuccess) return ::sil::cuda_fail(err_, #call); \
    } while (0)

// ---------------------------------------------------------------- launches

// Programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may start (barrier set-up) while the
// previous kernel on the stream drains; grid_dependency_wait() returns once
// that kernel has completed and its writes are visible, so every global
// access of the kernel comes after it.  Without the attribute both are no-ops.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Launch with the programmatic stream-serialization attribute, so that
// back-to-back runs overlap one kernel's drain with the next one's set-up.
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args... args)
{
    cudaLaunchConfig_t cfg {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

inline int64_t binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

inline int64_t ipow(int64_t b, int e)
{
    int64_t r = 1;
    for (int i = 0; i < e; ++i) r *= b;
    return r;
}

// ---------------------------------------------------------------- fields

// Field as the kernels see it (plain aggregate passed by value).
struct FieldView
{
    void* data;
    int32_t ndims;
    int32_t ncomp;
    int64_t front[kMaxDims];
    int64_t extent[kMaxDims];
    int64_t stride[kMaxDims];
    int64_t comp_stride;
};

FieldView to_view(sil_field const& f);
int64_t node_count(sil_field const& f);
sil_status check_field(sil_field const* f, char const* name, int expect_ncomp);
int form_dims(uint32_t mask, int ndims, int* dims);

// ---------------------------------------------------------------- chains

// A face of the boundary of a basis simplex, as a sampling rule: the sample
// is taken at node + offset, component `comp` of the lower tangent basis,
// with sign -1 when `negative`.
struct FaceRule
{
    int8_t offset[kMaxN];
    int8_t comp;
    int8_t negative;
};

// Sampling rules of d (clamped) or d^T (zero outside, shifted second half)
// for a k-form over n form dims: rules[c][f] for output component c.
struct CoboundaryRules
{
    int n;
    int k;
    int ncomp_in;
    int ncomp_out;
    int nfaces;
    FaceRule rule[kMaxComp][kMaxFaces];
};

CoboundaryRules make_rules(int n, int k, bool transposed);

// Diagonal Hodge star of an r-form over n dims: output component t (an
// (n-r)-combination) reads input component src[t] (the complementary
// r-combination) with sign sgn[t]; the factor is the product of the edge
// lengths along `num_mask[t]` divided by those along `den_mask[t]`.
struct StarRule
{
    int n;
    int r;
    int ncomp_out;
    int8_t src[kMaxComp];
    int8_t sgn[kMaxComp];
    uint8_t num_mask[kMaxComp];
    uint8_t den_mask[kMaxComp];
};

StarRule make_star(int n, int r);

// Lexicographic combinations of {0..n-1} of size k as bit masks; index =
// component id (matches SimiLie's antisymmetric-index memory order).
std::vector<uint32_t> combinations(int n, int k);

// ---------------------------------------------------------------- geometry

struct Geometry
{
    int n = 0;
    int64_t npoints[kMaxNHodge] = {0, 0, 0};
    int64_t front[kMaxNHodge] = {0, 0, 0};
    // Device arrays of length npoints + 2, index shifted by one: entry
    // [p + 1] is the edge length along the axis at node p (forward
    // difference, backward at the last node); the pads hold h = 1 and
    // inv_h = 0.
    double* h[kMaxNHodge] = {nullptr, nullptr, nullptr};
    double* inv_h[kMaxNHodge] = {nullptr, nullptr, nullptr};
    float* h32[kMaxNHodge] = {nullptr, nullptr, nullptr};
    float* inv_h32[kMaxNHodge] = {nullptr, nullptr, nullptr};
    std::vector<double> host_h[kMaxNHodge];
};

// Geometry view passed to kernels.
template <class T>
struct GeoView
{
    T const* h[kMaxNHodge];
    T const* inv_h[kMaxNHodge];
    int64_t front[kMaxNHodge];
    int64_t npoints[kMaxNHodge];
};

template <class T>
GeoView<T> geo_view(Geometry const& g);

// The divergence-gauge table of a 3D grid (8 doubles per node: the
// codifferential's coefficients E0[3], E1[3] read off parity probes, the
// node weight w, 0), as the linear 3D operator builds it; coords: host node
// coordinates per axis; ls: the device local-spacing table (x, y, z
// concatenated); probe (3 doubles per node) and out (1 per node) are
// scratch.  Defined in magnetostatics.cu.
sil_status divergence_gauge_table(int64_t nx, int64_t ny, int64_t nz, double const* const coords[3],
                                  double const* ls, double* gd, double* probe, double* out, cudaStream_t st);

// Stored Hodge tensors of a staged operator built from a (metric, position)
// pair, over the position lattice: h[0] the (k+1)-form star, h[1] the
// (n-k)-form star, h[2] the k-form star, h[3] the (n-k+1)-form star, with
// kin[w] their source ranks; data == nullptr where the operator needs none.
// Defined in staged_metric.cu.
struct StoredHodges
{
    int n = 0;
    int k = 0;
    int kin[4] = {0, 0, 0, 0};
    sil_field lattice {};
    sil_field h[4] {};
};

// Fills the tensors a Laplacian (laplacian = true: all four that its rank
// needs) or a codifferential (h[2], h[3]) stores; *mem owns them (cudaFree).
sil_status fill_stored_hodges(cudaStream_t stream, int n, int k, sil_field const& position, sil_field const* metric,
                              bool laplacian, void** mem, StoredHodges* out);
sil_status check_stored_laplacian(int n, int k, sil_field const* position, sil_field const* metric);
sil_status launch_stored_laplacian(cudaStream_t s, StoredHodges const& H, sil_field const* in, sil_field const* out);

} // namespace sil

struct sil_geometry_s
{
    sil::Geometry g;
};
