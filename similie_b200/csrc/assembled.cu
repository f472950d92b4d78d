// assembled.cu -- the magnetostatics operators as CSR matrices and the
// reference's preconditioner menu on them, with a preconditioned CG.
//
// Assembly (the reference's assemble_matrix_data, onelab_interface/
// magnetostatics_onelab.hpp:3120-3534 for 3D, 3554-3737 for 2D) probes the
// matrix-free operator: every row only touches columns in the 3x3 (2D) or
// 3x3x3 (3D, times 3 components) node neighbourhood, so columns coloured by
// their node coordinates mod 3 (and component) never share a row, and one
// apply per colour yields one entry of every row.  A first sweep over the
// colours marks the nonzero entries of each row in a bit mask (exact zeros
// are dropped, as the reference drops zero coefficients), a scan of the
// popcounts gives the row pointers, and a second sweep writes the entries
// in ascending column order.
//
// Preconditioners (minimize_strong_formulation_residual.hpp:53-63, defaults
// 61-75, construction 921-1026 through Ginkgo v1.11.0, whose source is not
// available here; each restates the published algorithm it names):
//   Jacobi              z = D^-1 r
//   SpdIsai             factorized sparse approximate inverse (Kolotilina &
//                       Yeremin): Z on the pattern of tril(A), row i solves
//                       A(P_i, P_i) y = e_i and is scaled by 1/sqrt(y_i);
//                       z = Z^T (Z r)
//   GeneralIsai         incomplete sparse approximate inverse (Anzt et al.
//                       2018): M on the pattern of A, (M A)(i, P_i) = e_i
//   SymmetricGaussSeidel, Ssor
//                       M = (D - w E) D^-1 (D - w F) / (w (2 - w)) with
//                       A = D - E - F (Saad, Iterative Methods for Sparse
//                       Linear Systems, sec. 10.2), w = 1 for Gauss-Seidel;
//                       the triangular solves run level by level (rows of a
//                       level depend only on earlier levels)
//   ChebyshevJacobi     k steps of the Chebyshev iteration on the Jacobi-
//                       preconditioned system, eigenvalue bounds [l, u], zero
//                       initial guess (Saad, Algorithm 12.1)
//   IrJacobi            k steps of x += w D^-1 (b - A x) from zero
// Every row-level expression keeps the order of the CPU restatement, so the
// preconditioners agree with it bit for bit on the same matrix.
#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "sil_internal.cuh"

struct sil_csr_s
{
    int64_t n = 0;
    int64_t nnz = 0;
    int32_t* ptr = nullptr;  // device, n + 1
    int32_t* col = nullptr;  // device, nnz
    double* val = nullptr;   // device, nnz
    ~sil_csr_s()
    {
        cudaFree(ptr);
        cudaFree(col);
        cudaFree(val);
    }
};

namespace sil {
namespace {

constexpr int kBlock = 256;
constexpr int kMaxIsai = 32;  // ISAI rows: at most this many pattern entries

unsigned grid_of(int64_t n)
{
    // initialised once, thread-safely (the nonlinear batches call this from
    // several host threads)
    static int const sms = [] {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        return count > 0 ? count : 148;
    }();
    int64_t const blocks = (n + kBlock - 1) / kBlock;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, 8 * sms)));
}

// ------------------------------------------------------------------ assembly

struct Probe
{
    int dim;  // 2 or 3
    int nx, ny, nz;
};

__device__ __forceinline__ int mod3_offset(int target, int at)
{
    int const d = ((target - at % 3) % 3 + 3) % 3;  // 0, 1, 2
    return d == 2 ? -1 : d;
}

// Colour of column c: 2D (i mod 3) + 3 (j mod 3); 3D comp + 3 ((i mod 3) +
// 3 (j mod 3) + 9 (k mod 3)).
__global__ void probe_kernel(Probe g, int color, double* probe, int64_t n)
{
    for (int64_t c = blockIdx.x * int64_t(kBlock) + threadIdx.x; c < n; c += int64_t(gridDim.x) * kBlock) {
        int col;
        if (g.dim == 2) {
            int const i = static_cast<int>(c % g.nx), j = static_cast<int>(c / g.nx);
            col = i % 3 + 3 * (j % 3);
        } else {
            int const node = static_cast<int>(c / 3), comp = static_cast<int>(c % 3);
            int const t = node / g.nx, i = node - t * g.nx, k = t / g.ny, j = t - k * g.ny;
            col = comp + 3 * (i % 3 + 3 * (j % 3) + 9 * (k % 3));
        }
        probe[c] = col == color ? 1.0 : 0.0;
    }
}

// The candidate column of row r in colour `color`: its slot (ascending
// column order within the neighbourhood) and index; false outside the grid.
__device__ __forceinline__ bool candidate(Probe const& g, int color, int64_t r, int* slot, int* column)
{
    if (g.dim == 2) {
        int const i = static_cast<int>(r % g.nx), j = static_cast<int>(r / g.nx);
        int const di = mod3_offset(color % 3, i), dj = mod3_offset(color / 3, j);
        if (i + di < 0 || i + di >= g.nx || j + dj < 0 || j + dj >= g.ny) return false;
        *slot = (dj + 1) * 3 + (di + 1);
        *column = (i + di) + g.nx * (j + dj);
        return true;
    }
    int const comp = color % 3, nc = color / 3;
    int const node = static_cast<int>(r / 3);
    int const t = node / g.nx, i = node - t * g.nx, k = t / g.ny, j = t - k * g.ny;
    int const di = mod3_offset(nc % 3, i), dj = mod3_offset((nc / 3) % 3, j), dk = mod3_offset(nc / 9, k);
    if (i + di < 0 || i + di >= g.nx || j + dj < 0 || j + dj >= g.ny || k + dk < 0 || k + dk >= g.nz) return false;
    *slot = (((dk + 1) * 3 + (dj + 1)) * 3 + (di + 1)) * 3 + comp;
    *column = 3 * ((i + di) + g.nx * ((j + dj) + g.ny * (k + dk))) + comp;
    return true;
}

__global__ void mark_kernel(Probe g, int color, double const* y, unsigned long long* mask, int64_t n)
{
    for (int64_t r = blockIdx.x * int64_t(kBlock) + threadIdx.x; r < n; r += int64_t(gridDim.x) * kBlock) {
        int slot, column;
        if (!candidate(g, color, r, &slot, &column) || y[r] == 0.0) continue;
        mask[2 * r + (slot >> 6)] |= 1ull << (slot & 63);
    }
}

__device__ __forceinline__ int popc_below(unsigned long long const* m, int slot)
{
    if (slot < 64) return __popcll(m[0] & ((1ull << slot) - 1ull));
    return __popcll(m[0]) + __popcll(m[1] & ((1ull << (slot - 64)) - 1ull));
}

__global__ void fill_kernel(Probe g, int color, double const* y, unsigned long long const* mask,
                            int32_t const* ptr, int32_t* col, double* val, int64_t n)
{
    for (int64_t r = blockIdx.x * int64_t(kBlock) + threadIdx.x; r < n; r += int64_t(gridDim.x) * kBlock) {
        int slot, column;
        if (!candidate(g, color, r, &slot, &column)) continue;
        unsigned long long const* m = mask + 2 * r;
        if (!((m[slot >> 6] >> (slot & 63)) & 1ull)) continue;
        int64_t const pos = ptr[r] + popc_below(m, slot);
        col[pos] = column;
        val[pos] = y[r];
    }
}

// Exclusive scan of per-row counts into ptr (one block of 1024 threads,
// contiguous chunks); *total = the sum (checked on the host against 2^31).
__global__ void __launch_bounds__(1024) scan_kernel(int64_t n, unsigned long long const* mask,
                                                    int32_t const* counts, int32_t* ptr, long long* total)
{
    __shared__ long long sums[1024];
    int const t = threadIdx.x;
    int64_t const chunk = (n + 1023) / 1024;
    int64_t const lo = std::min<int64_t>(n, t * chunk), hi = std::min<int64_t>(n, lo + chunk);
    auto count = [&](int64_t i) -> long long {
        if (mask != nullptr) return __popcll(mask[2 * i]) + __popcll(mask[2 * i + 1]);
        return counts[i];
    };
    long long s = 0;
    for (int64_t i = lo; i < hi; ++i) s += count(i);
    sums[t] = s;
    __syncthreads();
    if (t == 0) {
        long long acc = 0;
        for (int u = 0; u < 1024; ++u) {
            long long const v = sums[u];
            sums[u] = acc;
            acc += v;
        }
        *total = acc;
        ptr[n] = static_cast<int32_t>(acc);
    }
    __syncthreads();
    long long acc = sums[t];
    for (int64_t i = lo; i < hi; ++i) {
        ptr[i] = static_cast<int32_t>(acc);
        acc += count(i);
    }
}

__global__ void spmv_kernel(int64_t n, int32_t const* ptr, int32_t const* col, double const* val, double const* x,
                            double* y)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double s = 0.0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

struct DevBuf
{
    void* p = nullptr;
    ~DevBuf() { cudaFree(p); }
};

template <class Apply>
sil_status assemble(cudaStream_t s, Probe g, int64_t n, int ncolors, Apply const& apply, sil_csr* out)
{
    if (n >= (int64_t(1) << 31)) return fail(SIL_ERR_INVALID, "assemble: fewer than 2^31 rows supported");
    DevBuf work;
    size_t const vb = (static_cast<size_t>(n) * sizeof(double) + 255) / 256 * 256;
    size_t const mb = static_cast<size_t>(n) * 2 * sizeof(unsigned long long);
    SIL_CUDA_CHECK(cudaMalloc(&work.p, 2 * vb + mb + 256));
    double* probe = static_cast<double*>(work.p);
    double* y = reinterpret_cast<double*>(static_cast<char*>(work.p) + vb);
    auto* mask = reinterpret_cast<unsigned long long*>(static_cast<char*>(work.p) + 2 * vb);
    auto* total = reinterpret_cast<long long*>(static_cast<char*>(work.p) + 2 * vb + mb);
    SIL_CUDA_CHECK(cudaMemsetAsync(mask, 0, mb, s));
    unsigned const G = grid_of(n);
    for (int c = 0; c < ncolors; ++c) {
        probe_kernel<<<G, kBlock, 0, s>>>(g, c, probe, n);
        if (sil_status st = apply(probe, y); st != SIL_OK) return st;
        mark_kernel<<<G, kBlock, 0, s>>>(g, c, y, mask, n);
    }
    auto m = std::make_unique<sil_csr_s>();
    m->n = n;
    SIL_CUDA_CHECK(cudaMalloc(&m->ptr, static_cast<size_t>(n + 1) * sizeof(int32_t)));
    scan_kernel<<<1, 1024, 0, s>>>(n, mask, nullptr, m->ptr, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    long long nnz = 0;
    SIL_CUDA_CHECK(cudaMemcpyAsync(&nnz, total, sizeof(nnz), cudaMemcpyDeviceToHost, s));
    SIL_CUDA_CHECK(cudaStreamSynchronize(s));
    if (nnz >= (1ll << 31)) return fail(SIL_ERR_INVALID, "assemble: fewer than 2^31 nonzeros supported");
    m->nnz = nnz;
    SIL_CUDA_CHECK(cudaMalloc(&m->col, std::max<size_t>(1, static_cast<size_t>(nnz)) * sizeof(int32_t)));
    SIL_CUDA_CHECK(cudaMalloc(&m->val, std::max<size_t>(1, static_cast<size_t>(nnz)) * sizeof(double)));
    for (int c = 0; c < ncolors; ++c) {
        probe_kernel<<<G, kBlock, 0, s>>>(g, c, probe, n);
        if (sil_status st = apply(probe, y); st != SIL_OK) return st;
        fill_kernel<<<G, kBlock, 0, s>>>(g, c, y, mask, m->ptr, m->col, m->val, n);
    }
    SIL_CUDA_CHECK(cudaGetLastError());
    SIL_CUDA_CHECK(cudaStreamSynchronize(s));
    *out = m.release();
    return SIL_OK;
}

// ------------------------------------------------------------------ preconditioners

struct CgState
{
    double rz, pq, alpha, beta, bn, rn;
    int done, iters;
};

__device__ __forceinline__ bool skip(CgState const* st) { return st != nullptr && st->done; }

__global__ void diag_kernel(int64_t n, int32_t const* ptr, int32_t const* col, double const* val, double* diag,
                            double* dinv)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double d = 0.0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
            if (col[k] == i) {
                d = val[k];
                break;
            }
        diag[i] = d;
        dinv[i] = 1.0 / d;
    }
}

__device__ __forceinline__ double csr_at(int32_t const* ptr, int32_t const* col, double const* val, int r, int c)
{
    for (int32_t k = ptr[r]; k < ptr[r + 1]; ++k)
        if (col[k] == c) return val[k];
    return 0.0;
}

// One ISAI row per thread: the pattern P (the factor's columns of row i),
// G = A(P, P) (SpdIsai) or A(P, P)^T (GeneralIsai), G y = e_t by Gaussian
// elimination with partial pivoting, then the row's values.  *bad is set if
// a system is singular or a row is longer than kMaxIsai.
__global__ void isai_kernel(int64_t n, int spd, int32_t const* ptr, int32_t const* col, double const* val,
                            int32_t const* mptr, int32_t const* mcol, double* mval, int* bad)
{
    double G[kMaxIsai * kMaxIsai];
    double y[kMaxIsai];
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        int32_t const b0 = mptr[i];
        int const m = mptr[i + 1] - b0;
        if (m > kMaxIsai || m <= 0) {
            atomicExch(bad, 1);
            continue;
        }
        int t = 0;
        for (int a = 0; a < m; ++a) {
            int const pa = mcol[b0 + a];
            if (pa == i) t = a;
            for (int b = 0; b < m; ++b) {
                int const pb = mcol[b0 + b];
                G[a * m + b] = spd ? csr_at(ptr, col, val, pa, pb) : csr_at(ptr, col, val, pb, pa);
            }
        }
        for (int a = 0; a < m; ++a) y[a] = 0.0;
        y[t] = 1.0;
        bool ok = true;
        for (int c = 0; c < m && ok; ++c) {
            int p = c;
            for (int r = c + 1; r < m; ++r)
                if (fabs(G[r * m + c]) > fabs(G[p * m + c])) p = r;
            if (G[p * m + c] == 0.0) {
                ok = false;
                break;
            }
            if (p != c) {
                for (int k = 0; k < m; ++k) {
                    double const tmp = G[c * m + k];
                    G[c * m + k] = G[p * m + k];
                    G[p * m + k] = tmp;
                }
                double const tmp = y[c];
                y[c] = y[p];
                y[p] = tmp;
            }
            for (int r = c + 1; r < m; ++r) {
                double const f = G[r * m + c] / G[c * m + c];
                for (int k = c; k < m; ++k) G[r * m + k] -= f * G[c * m + k];
                y[r] -= f * y[c];
            }
        }
        if (!ok) {
            atomicExch(bad, 1);
            continue;
        }
        for (int r = m - 1; r >= 0; --r) {
            double s = y[r];
            for (int k = r + 1; k < m; ++k) s -= G[r * m + k] * y[k];
            y[r] = s / G[r * m + r];
        }
        double const scale = spd ? 1.0 / sqrt(y[t]) : 1.0;
        for (int a = 0; a < m; ++a) mval[b0 + a] = spd ? y[a] * scale : y[a];
    }
}

__global__ void gather_kernel(int64_t n, int32_t const* perm, double const* src, double* dst)
{
    for (int64_t e = blockIdx.x * int64_t(kBlock) + threadIdx.x; e < n; e += int64_t(gridDim.x) * kBlock)
        dst[perm[e]] = src[e];
}

__global__ void spmv_pc_kernel(int64_t n, int32_t const* ptr, int32_t const* col, double const* val,
                               double const* x, double* y, CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double s = 0.0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

__global__ void copy_kernel(int64_t n, double const* r, double* z, CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) z[i] = r[i];
}

// z = w * (dinv r) (w = 1: Jacobi; the first IR step)
__global__ void jacobi_kernel(int64_t n, double w, bool scaled, double const* dinv, double const* r, double* z,
                              CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        z[i] = scaled ? w * (dinv[i] * r[i]) : dinv[i] * r[i];
}

// z += w (dinv (r - ax))
__global__ void ir_step_kernel(int64_t n, double w, double const* dinv, double const* r, double const* ax, double* z,
                               CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        z[i] += w * (dinv[i] * (r[i] - ax[i]));
}

// d = dinv r / theta, z = d
__global__ void cheb_init_kernel(int64_t n, double theta, double const* dinv, double const* r, double* d, double* z,
                                 CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double const v = dinv[i] * r[i] / theta;
        d[i] = v;
        z[i] = v;
    }
}

// d = c1 d + c2 (dinv (r - ax)), z += d
__global__ void cheb_step_kernel(int64_t n, double c1, double c2, double const* dinv, double const* r,
                                 double const* ax, double* d, double* z, CgState const* st)
{
    if (skip(st)) return;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double const res = r[i] - ax[i];
        double const v = c1 * d[i] + c2 * (dinv[i] * res);
        d[i] = v;
        z[i] += v;
    }
}

// Forward SSOR sweep over the rows of one level:
// y_i = (c r_i - sum_{j<i} w a_ij y_j) / a_ii
__global__ void ssor_fwd_kernel(int count, int32_t const* rows, int32_t const* ptr, int32_t const* col,
                                double const* val, double const* diag, double w, double c, double const* r,
                                double* y, CgState const* st)
{
    if (skip(st)) return;
    int const t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= count) return;
    int const i = rows[t];
    double s = c * r[i];
    for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
        if (col[k] < i) s -= w * val[k] * y[col[k]];
    y[i] = s / diag[i];
}

// Backward sweep: z_i = (a_ii y_i - sum_{j>i} w a_ij z_j) / a_ii
__global__ void ssor_bwd_kernel(int count, int32_t const* rows, int32_t const* ptr, int32_t const* col,
                                double const* val, double const* diag, double w, double const* y, double* z,
                                CgState const* st)
{
    if (skip(st)) return;
    int const t = blockIdx.x * kBlock + threadIdx.x;
    if (t >= count) return;
    int const i = rows[t];
    double s = diag[i] * y[i];
    for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
        if (col[k] > i) s -= w * val[k] * z[col[k]];
    z[i] = s / diag[i];
}

// One launch per triangular sweep of SSOR / symmetric Gauss-Seidel, in place
// of one launch per level: a single CTA walks the levels in order, its
// threads sharing each level's rows, with a barrier between levels (a
// level's rows read only rows of earlier levels, which the barrier makes
// visible within the CTA).  The sweeps are a chain of short levels (a 2D
// grid of n^2 nodes has 2n - 1), so one CTA holds a level's rows and the
// barrier costs far less than a launch.  Each row is the expression of the
// level kernels, so the values are the same.
constexpr int kSweepThreads = 1024;

template <bool FWD>
__global__ void __launch_bounds__(kSweepThreads) ssor_sweep_kernel(int nlev, int32_t const* lev, int32_t const* rows,
                                                                    int32_t const* ptr, int32_t const* col,
                                                                    double const* val, double const* diag, double w,
                                                                    double c, double const* in, double* out,
                                                                    CgState const* st)
{
    if (skip(st)) return;
    for (int l = 0; l < nlev; ++l) {
        int const end = lev[l + 1];
        for (int pos = lev[l] + static_cast<int>(threadIdx.x); pos < end; pos += kSweepThreads) {
            int const i = rows[pos];
            // forward: y_i = (c r_i - sum_{j<i} w a_ij y_j) / a_ii
            // backward: z_i = (a_ii y_i - sum_{j>i} w a_ij z_j) / a_ii
            double s = FWD ? c * in[i] : diag[i] * in[i];
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
                int const j = col[k];
                if (FWD ? j < i : j > i) s -= w * val[k] * out[j];
            }
            out[i] = s / diag[i];
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace sil

struct sil_csr_precond_s
{
    sil_csr_s const* A = nullptr;
    sil_menu_settings cfg {};
    int64_t n = 0;
    double* diag = nullptr;  // device, n
    double* dinv = nullptr;
    double* scratch = nullptr;  // device, 3 n (SSOR y, Chebyshev d / res, SpdIsai t)
    // ISAI factor (Z lower for SpdIsai, M for GeneralIsai) and Z^T
    int32_t *mptr = nullptr, *mcol = nullptr, *tptr = nullptr, *tcol = nullptr;
    double *mval = nullptr, *tval = nullptr;
    // SSOR levels: rows in level order, level offsets on the host
    int32_t *fwd_rows = nullptr, *bwd_rows = nullptr;
    std::vector<int32_t> fwd_lev, bwd_lev;
    // single-launch sweeps: the level offsets on the device
    int32_t *fwd_lev_d = nullptr, *bwd_lev_d = nullptr;
    ~sil_csr_precond_s()
    {
        for (void* p : {static_cast<void*>(diag), static_cast<void*>(dinv), static_cast<void*>(scratch),
                        static_cast<void*>(mptr), static_cast<void*>(mcol), static_cast<void*>(tptr),
                        static_cast<void*>(tcol), static_cast<void*>(mval), static_cast<void*>(tval),
                        static_cast<void*>(fwd_rows), static_cast<void*>(bwd_rows), static_cast<void*>(fwd_lev_d),
                        static_cast<void*>(bwd_lev_d)})
            cudaFree(p);
    }
};

namespace sil {
namespace {

sil_menu_settings with_defaults(sil_menu_settings c)
{
    if (c.sor_relaxation_factor == 0.0) c.sor_relaxation_factor = 1.2;
    if (c.chebyshev_iterations <= 0) c.chebyshev_iterations = 8;
    if (c.chebyshev_lower_bound == 0.0) c.chebyshev_lower_bound = 0.05;
    if (c.chebyshev_upper_bound == 0.0) c.chebyshev_upper_bound = 1.5;
    if (c.ir_iterations <= 0) c.ir_iterations = 8;
    if (c.ir_relaxation_factor == 0.0) c.ir_relaxation_factor = 1.0;
    return c;
}

// z = M^-1 r on stream s (st: the CG state, whose done flag skips the work).
void precond_launch(sil_csr_precond_s const& P, cudaStream_t s, double const* r, double* z, CgState const* st)
{
    sil_csr_s const& A = *P.A;
    int64_t const n = P.n;
    unsigned const G = grid_of(n);
    sil_menu_settings const& c = P.cfg;
    switch (c.kind) {
    case SIL_PC_IDENTITY:
        copy_kernel<<<G, kBlock, 0, s>>>(n, r, z, st);
        return;
    case SIL_PC_JACOBI:
        jacobi_kernel<<<G, kBlock, 0, s>>>(n, 1.0, false, P.dinv, r, z, st);
        return;
    case SIL_PC_SPD_ISAI:
        spmv_pc_kernel<<<G, kBlock, 0, s>>>(n, P.mptr, P.mcol, P.mval, r, P.scratch, st);
        spmv_pc_kernel<<<G, kBlock, 0, s>>>(n, P.tptr, P.tcol, P.tval, P.scratch, z, st);
        return;
    case SIL_PC_GENERAL_ISAI:
        spmv_pc_kernel<<<G, kBlock, 0, s>>>(n, P.mptr, P.mcol, P.mval, r, z, st);
        return;
    case SIL_PC_SYMMETRIC_GAUSS_SEIDEL:
    case SIL_PC_SSOR: {
        double const w = c.kind == SIL_PC_SSOR ? c.sor_relaxation_factor : 1.0;
        double const cw = w * (2.0 - w);
        double* y = P.scratch;
        if (P.fwd_lev_d != nullptr) {
            ssor_sweep_kernel<true><<<1, kSweepThreads, 0, s>>>(static_cast<int>(P.fwd_lev.size()) - 1, P.fwd_lev_d,
                                                                 P.fwd_rows, A.ptr, A.col, A.val, P.diag, w, cw, r, y, st);
            ssor_sweep_kernel<false><<<1, kSweepThreads, 0, s>>>(static_cast<int>(P.bwd_lev.size()) - 1, P.bwd_lev_d,
                                                                  P.bwd_rows, A.ptr, A.col, A.val, P.diag, w, 0.0, y, z,
                                                                  st);
            return;
        }
        for (size_t l = 0; l + 1 < P.fwd_lev.size(); ++l) {
            int const cnt = P.fwd_lev[l + 1] - P.fwd_lev[l];
            ssor_fwd_kernel<<<(cnt + kBlock - 1) / kBlock, kBlock, 0, s>>>(cnt, P.fwd_rows + P.fwd_lev[l], A.ptr,
                                                                          A.col, A.val, P.diag, w, cw, r, y, st);
        }
        for (size_t l = 0; l + 1 < P.bwd_lev.size(); ++l) {
            int const cnt = P.bwd_lev[l + 1] - P.bwd_lev[l];
            ssor_bwd_kernel<<<(cnt + kBlock - 1) / kBlock, kBlock, 0, s>>>(cnt, P.bwd_rows + P.bwd_lev[l], A.ptr,
                                                                          A.col, A.val, P.diag, w, y, z, st);
        }
        return;
    }
    case SIL_PC_CHEBYSHEV_JACOBI: {
        double const theta = 0.5 * (c.chebyshev_upper_bound + c.chebyshev_lower_bound);
        double const delta = 0.5 * (c.chebyshev_upper_bound - c.chebyshev_lower_bound);
        double const sigma = theta / delta;
        double rho = 1.0 / sigma;
        double* d = P.scratch;
        double* ax = P.scratch + n;
        cheb_init_kernel<<<G, kBlock, 0, s>>>(n, theta, P.dinv, r, d, z, st);
        for (int it = 1; it < c.chebyshev_iterations; ++it) {
            spmv_pc_kernel<<<G, kBlock, 0, s>>>(n, A.ptr, A.col, A.val, z, ax, st);
            double const rho1 = 1.0 / (2.0 * sigma - rho);
            cheb_step_kernel<<<G, kBlock, 0, s>>>(n, rho1 * rho, 2.0 * rho1 / delta, P.dinv, r, ax, d, z, st);
            rho = rho1;
        }
        return;
    }
    case SIL_PC_IR_JACOBI: {
        double* ax = P.scratch;
        jacobi_kernel<<<G, kBlock, 0, s>>>(n, c.ir_relaxation_factor, true, P.dinv, r, z, st);
        for (int it = 1; it < c.ir_iterations; ++it) {
            spmv_pc_kernel<<<G, kBlock, 0, s>>>(n, A.ptr, A.col, A.val, z, ax, st);
            ir_step_kernel<<<G, kBlock, 0, s>>>(n, c.ir_relaxation_factor, P.dinv, r, ax, z, st);
        }
        return;
    }
    default:
        return;
    }
}

// Level sets of the forward (lower) and backward (upper) triangular solves:
// a row's level is one more than the largest level among the rows it reads.
void levels(std::vector<int32_t> const& ptr, std::vector<int32_t> const& col, bool lower, std::vector<int32_t>& rows,
            std::vector<int32_t>& lev_ptr)
{
    int64_t const n = static_cast<int64_t>(ptr.size()) - 1;
    std::vector<int32_t> level(n, 0);
    int32_t top = 0;
    for (int64_t t = 0; t < n; ++t) {
        int64_t const i = lower ? t : n - 1 - t;
        int32_t l = 0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            int32_t const j = col[k];
            if (lower ? j < i : j > i) l = std::max(l, level[j] + 1);
        }
        level[i] = l;
        top = std::max(top, l);
    }
    lev_ptr.assign(top + 2, 0);
    for (int64_t i = 0; i < n; ++i) ++lev_ptr[level[i] + 1];
    for (int32_t l = 0; l <= top; ++l) lev_ptr[l + 1] += lev_ptr[l];
    rows.assign(n, 0);
    std::vector<int32_t> fill(lev_ptr.begin(), lev_ptr.end() - 1);
    for (int64_t i = 0; i < n; ++i) rows[fill[level[i]]++] = static_cast<int32_t>(i);
}

template <class T>
sil_status upload(T** dst, std::vector<T> const& src, cudaStream_t s)
{
    SIL_CUDA_CHECK(cudaMalloc(dst, std::max<size_t>(1, src.size()) * sizeof(T)));
    if (!src.empty())
        SIL_CUDA_CHECK(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return SIL_OK;
}

// ------------------------------------------------------------------ CG

__device__ __forceinline__ double block_sum(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
    return t;
}

__device__ __forceinline__ double sum_parts(double const* part, int nparts, double* red)
{
    double v = 0.0;
    for (int b = threadIdx.x; b < nparts; b += kBlock) v += part[b];
    return block_sum(v, red);
}

// x = 0, r = b, partial b.b
__global__ void cg_start_kernel(int64_t n, double const* b, double* x, double* r, double* part)
{
    __shared__ double red[kBlock / 32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double const v = b[i];
        x[i] = 0.0;
        r[i] = v;
        acc += v * v;
    }
    double const t = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void cg_init_kernel(double const* part, int nparts, CgState* st, int max_iter)
{
    __shared__ double red[kBlock / 32];
    double const t = sum_parts(part, nparts, red);
    if (threadIdx.x == 0) {
        st->bn = sqrt(t);
        st->rn = st->bn;
        st->iters = 0;
        st->done = (max_iter <= 0 || st->bn == 0.0) ? 1 : 0;
    }
}

// partial a.b (skipped when done)
__global__ void dot_kernel(int64_t n, double const* a, double const* b, double* part, CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (skip(st)) return;
    double acc = 0.0;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        acc += a[i] * b[i];
    double const t = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// p = z (first) or p = z + beta p with beta = (r.z) / rz; every block sums
// the r.z partials itself in the same fixed order, and rz is replaced by the
// next kernel (cg_rz_kernel), after every block has read it.
__global__ void cg_direction_kernel(int64_t n, double const* part, int nparts, double const* z, double* p,
                                    CgState const* st, int first)
{
    __shared__ double red[kBlock / 32];
    __shared__ double beta;
    if (st->done) return;
    double const t = sum_parts(part, nparts, red);
    if (threadIdx.x == 0) beta = first ? 0.0 : t / st->rz;
    __syncthreads();
    double const bt = beta;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        p[i] = first ? z[i] : z[i] + bt * p[i];
}

__global__ void cg_rz_kernel(double const* part, int nparts, CgState* st)
{
    __shared__ double red[kBlock / 32];
    if (st->done) return;
    double const t = sum_parts(part, nparts, red);
    if (threadIdx.x == 0) st->rz = t;
}

// q = A p, partial p.q
__global__ void cg_spmv_kernel(int64_t n, int32_t const* ptr, int32_t const* col, double const* val, double const* p,
                               double* q, double* part, CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (skip(st)) return;
    double acc = 0.0;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        double s = 0.0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * p[col[k]];
        q[i] = s;
        acc += p[i] * s;
    }
    double const t = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void cg_alpha_kernel(double const* part, int nparts, CgState* st)
{
    __shared__ double red[kBlock / 32];
    if (st->done) return;
    double const t = sum_parts(part, nparts, red);
    if (threadIdx.x == 0) {
        st->pq = t;
        st->alpha = st->rz / t;
    }
}

// x += alpha p, r -= alpha q, partial r.r
__global__ void cg_update_kernel(int64_t n, double* x, double* r, double const* p, double const* q, double* part,
                                 CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (skip(st)) return;
    double const alpha = st->alpha;
    double acc = 0.0;
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock) {
        x[i] += alpha * p[i];
        double const v = r[i] - alpha * q[i];
        r[i] = v;
        acc += v * v;
    }
    double const t = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void cg_check_kernel(double const* part, int nparts, CgState* st, double tol, int max_iter)
{
    __shared__ double red[kBlock / 32];
    if (st->done) return;
    double const t = sum_parts(part, nparts, red);
    if (threadIdx.x == 0) {
        st->iters += 1;
        st->rn = sqrt(t);
        if (st->rn <= tol * st->bn || st->iters >= max_iter || !isfinite(st->rn)) st->done = 1;
    }
}

}  // namespace
}  // namespace sil

namespace sil {
namespace {

// ------------------------------------------------------------------ Krylov menu
//
// Host-driven restatements of the published methods (the same steps as the
// CPU restatement): vectors on the device, scalars on the host, every dot
// product reduced from fixed per-block partials in a fixed order.

__global__ void axpy_k(int64_t n, double a, double const* x, double* y)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        y[i] += a * x[i];
}

// out = a x + b y
__global__ void lin2_k(int64_t n, double a, double const* x, double b, double const* y, double* out)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        out[i] = a * x[i] + b * y[i];
}

__global__ void scale_k(int64_t n, double a, double const* x, double* out)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        out[i] = x[i] / a;
}

// BiCGSTAB direction: p = r + beta (p - omega v)
__global__ void bicg_p_k(int64_t n, double beta, double omega, double const* r, double const* v, double* p)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        p[i] = r[i] + beta * (p[i] - omega * v[i]);
}

// MINRES direction: d = (w - r3 d_older - r2 d_old) / r1
__global__ void minres_d_k(int64_t n, double r1, double r2, double r3, double const* w, double const* d_older,
                           double const* d_old, double* d)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        d[i] = (w[i] - r3 * d_older[i] - r2 * d_old[i]) / r1;
}

// MINRES Lanczos vector: v_new = q - a v - b v_old
__global__ void lanczos_k(int64_t n, double a, double b, double const* q, double const* v, double const* v_old,
                          double* v_new)
{
    for (int64_t i = blockIdx.x * int64_t(kBlock) + threadIdx.x; i < n; i += int64_t(gridDim.x) * kBlock)
        v_new[i] = q[i] - a * v[i] - b * v_old[i];
}

class Krylov
{
public:
    Krylov(cudaStream_t s, sil_csr_s const& A, sil_csr_precond_s const& P)
        : s_(s), A_(A), P_(P), n_(A.n), G_(grid_of(A.n)), hpart_(G_)
    {
    }
    ~Krylov() { cudaFree(buf_); }

    // device vectors, zeroed
    sil_status alloc(int count)
    {
        size_t const vb = (static_cast<size_t>(n_) * sizeof(double) + 255) / 256 * 256;
        size_t const pb = (static_cast<size_t>(G_) * sizeof(double) + 255) / 256 * 256;
        SIL_CUDA_CHECK(cudaMalloc(&buf_, count * vb + pb));
        SIL_CUDA_CHECK(cudaMemsetAsync(buf_, 0, count * vb + pb, s_));
        for (int k = 0; k < count; ++k) v_.push_back(reinterpret_cast<double*>(static_cast<char*>(buf_) + k * vb));
        part_ = reinterpret_cast<double*>(static_cast<char*>(buf_) + count * vb);
        return SIL_OK;
    }
    double* vec(int k) const { return v_[k]; }
    int64_t n() const { return n_; }

    sil_status dot(double const* a, double const* b, double* out)
    {
        dot_kernel<<<G_, kBlock, 0, s_>>>(n_, a, b, part_, nullptr);
        SIL_CUDA_CHECK(cudaGetLastError());
        SIL_CUDA_CHECK(cudaMemcpyAsync(hpart_.data(), part_, G_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
        SIL_CUDA_CHECK(cudaStreamSynchronize(s_));
        double t = 0.0;
        for (double v : hpart_) t += v;
        *out = t;
        return SIL_OK;
    }
    sil_status norm(double const* a, double* out)
    {
        double t = 0.0;
        if (sil_status st = dot(a, a, &t); st != SIL_OK) return st;
        *out = std::sqrt(t);
        return SIL_OK;
    }
    void spmv(double const* x, double* y) { spmv_kernel<<<G_, kBlock, 0, s_>>>(n_, A_.ptr, A_.col, A_.val, x, y); }
    void precond(double const* r, double* z) { precond_launch(P_, s_, r, z, nullptr); }
    void axpy(double a, double const* x, double* y) { axpy_k<<<G_, kBlock, 0, s_>>>(n_, a, x, y); }
    void lin2(double a, double const* x, double b, double const* y, double* out)
    {
        lin2_k<<<G_, kBlock, 0, s_>>>(n_, a, x, b, y, out);
    }
    void copy(double const* x, double* y)
    {
        cudaMemcpyAsync(y, x, static_cast<size_t>(n_) * sizeof(double), cudaMemcpyDeviceToDevice, s_);
    }
    void divide(double const* x, double a, double* out) { scale_k<<<G_, kBlock, 0, s_>>>(n_, a, x, out); }
    unsigned grid() const { return G_; }
    cudaStream_t stream() const { return s_; }

private:
    cudaStream_t s_;
    sil_csr_s const& A_;
    sil_csr_precond_s const& P_;
    int64_t n_;
    unsigned G_;
    void* buf_ = nullptr;
    std::vector<double*> v_;
    double* part_ = nullptr;
    std::vector<double> hpart_;
};

#define KRY_CHECK(call)                                    \
    do {                                                   \
        if (sil_status const kst_ = (call); kst_ != SIL_OK) \
            return kst_;                                   \
    } while (0)

// Each returns the iterations in *its and the last residual norm in *rn.
sil_status run_fcg(Krylov& K, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    KRY_CHECK(K.alloc(6));
    double *r = K.vec(0), *z = K.vec(1), *p = K.vec(2), *q = K.vec(3), *r_old = K.vec(4), *t = K.vec(5);
    K.copy(b, r);
    K.precond(r, z);
    K.copy(z, p);
    double rz = 0.0;
    KRY_CHECK(K.dot(r, z, &rz));
    KRY_CHECK(K.norm(b, rn));
    int it = 0;
    while (it < max_iter) {
        K.spmv(p, q);
        double pq = 0.0;
        KRY_CHECK(K.dot(p, q, &pq));
        double const alpha = rz / pq;
        K.axpy(alpha, p, x);
        K.copy(r, r_old);
        K.axpy(-alpha, q, r);
        ++it;
        KRY_CHECK(K.norm(r, rn));
        if (!(*rn > target)) break;
        K.precond(r, z);
        K.lin2(1.0, r, -1.0, r_old, t);
        double num = 0.0;
        KRY_CHECK(K.dot(z, t, &num));
        double const beta = num / rz;
        KRY_CHECK(K.dot(r, z, &rz));
        K.lin2(1.0, z, beta, p, p);
    }
    *its = it;
    return SIL_OK;
}

sil_status run_minres(Krylov& K, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    KRY_CHECK(K.alloc(12));
    double *v_old = K.vec(0), *v = K.vec(1), *w = K.vec(2), *v_new = K.vec(3), *w_new = K.vec(4), *q = K.vec(5);
    double *d_older = K.vec(6), *d_old = K.vec(7), *d = K.vec(8), *t = K.vec(9);
    K.copy(b, v);
    K.precond(v, w);
    double vw = 0.0;
    KRY_CHECK(K.dot(v, w, &vw));
    double beta = std::sqrt(vw), beta_prev = 1.0, eta = beta;
    double c_old = 1.0, s_old = 0.0, c = 1.0, s = 0.0;
    KRY_CHECK(K.norm(b, rn));
    int it = 0;
    while (it < max_iter && beta > 0.0) {
        K.divide(w, beta, w);
        K.spmv(w, q);
        double alpha = 0.0;
        KRY_CHECK(K.dot(w, q, &alpha));
        lanczos_k<<<K.grid(), kBlock, 0, K.stream()>>>(K.n(), alpha / beta, beta / beta_prev, q, v, v_old, v_new);
        K.precond(v_new, w_new);
        double vv = 0.0;
        KRY_CHECK(K.dot(v_new, w_new, &vv));
        double const beta_new = std::sqrt(std::max(0.0, vv));
        double const delta = c * alpha - c_old * s * beta;
        double const rho2 = s * alpha + c_old * c * beta;
        double const rho3 = s_old * beta;
        double const rho1 = std::sqrt(delta * delta + beta_new * beta_new);
        double const c_new = delta / rho1, s_new = beta_new / rho1;
        minres_d_k<<<K.grid(), kBlock, 0, K.stream()>>>(K.n(), rho1, rho2, rho3, w, d_older, d_old, d);
        K.axpy(c_new * eta, d, x);
        eta = -s_new * eta;
        K.copy(d_old, d_older);
        K.copy(d, d_old);
        K.copy(v, v_old);
        K.copy(v_new, v);
        K.copy(w_new, w);
        beta_prev = beta;
        beta = beta_new;
        c_old = c;
        s_old = s;
        c = c_new;
        s = s_new;
        ++it;
        K.spmv(x, t);
        K.lin2(1.0, b, -1.0, t, t);
        KRY_CHECK(K.norm(t, rn));
        if (!(*rn > target)) break;
    }
    *its = it;
    return SIL_OK;
}

sil_status run_gmres(Krylov& K, int m, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    KRY_CHECK(K.alloc(m + 5));
    double *r = K.vec(m + 1), *z = K.vec(m + 2), *u = K.vec(m + 3), *t = K.vec(m + 4);
    std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    K.copy(b, r);
    KRY_CHECK(K.norm(b, rn));
    int it = 0;
    while (it < max_iter) {
        double beta = 0.0;
        KRY_CHECK(K.norm(r, &beta));
        if (!(beta > target)) {
            *rn = beta;
            break;
        }
        K.divide(r, beta, K.vec(0));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        bool done = false;
        for (; k < m && it < max_iter; ++k) {
            K.precond(K.vec(k), z);
            K.spmv(z, u);
            for (int j = 0; j <= k; ++j) {
                double h = 0.0;
                KRY_CHECK(K.dot(u, K.vec(j), &h));
                H[j * m + k] = h;
                K.axpy(-h, K.vec(j), u);
            }
            double hn = 0.0;
            KRY_CHECK(K.norm(u, &hn));
            H[(k + 1) * m + k] = hn;
            if (hn != 0.0) K.divide(u, hn, K.vec(k + 1));
            for (int j = 0; j < k; ++j) {
                double const a = H[j * m + k], bb = H[(j + 1) * m + k];
                H[j * m + k] = cs[j] * a + sn[j] * bb;
                H[(j + 1) * m + k] = -sn[j] * a + cs[j] * bb;
            }
            double const a = H[k * m + k], bb = H[(k + 1) * m + k];
            double const den = std::sqrt(a * a + bb * bb);
            cs[k] = a / den;
            sn[k] = bb / den;
            H[k * m + k] = den;
            H[(k + 1) * m + k] = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            ++it;
            *rn = std::fabs(g[k + 1]);
            if (!(*rn > target)) {
                ++k;
                done = true;
                break;
            }
        }
        for (int j = k - 1; j >= 0; --j) {
            double acc = g[j];
            for (int l = j + 1; l < k; ++l) acc -= H[j * m + l] * y[l];
            y[j] = acc / H[j * m + j];
        }
        cudaMemsetAsync(u, 0, static_cast<size_t>(K.n()) * sizeof(double), K.stream());
        for (int j = 0; j < k; ++j) K.axpy(y[j], K.vec(j), u);
        K.precond(u, z);
        K.axpy(1.0, z, x);
        K.spmv(x, t);
        K.lin2(1.0, b, -1.0, t, r);
        if (done) break;
    }
    *its = it;
    return SIL_OK;
}

sil_status run_bicgstab(Krylov& K, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    KRY_CHECK(K.alloc(8));
    double *r = K.vec(0), *r0 = K.vec(1), *v = K.vec(2), *p = K.vec(3), *ph = K.vec(4), *sv = K.vec(5),
           *sh = K.vec(6), *tv = K.vec(7);
    K.copy(b, r);
    K.copy(b, r0);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    KRY_CHECK(K.norm(b, rn));
    int it = 0;
    while (it < max_iter) {
        double rho_new = 0.0;
        KRY_CHECK(K.dot(r0, r, &rho_new));
        double const beta = (rho_new / rho) * (alpha / omega);
        bicg_p_k<<<K.grid(), kBlock, 0, K.stream()>>>(K.n(), beta, omega, r, v, p);
        K.precond(p, ph);
        K.spmv(ph, v);
        double r0v = 0.0;
        KRY_CHECK(K.dot(r0, v, &r0v));
        alpha = rho_new / r0v;
        K.lin2(1.0, r, -alpha, v, sv);
        ++it;
        double sn = 0.0;
        KRY_CHECK(K.norm(sv, &sn));
        if (!(sn > target)) {
            K.axpy(alpha, ph, x);
            *rn = sn;
            break;
        }
        K.precond(sv, sh);
        K.spmv(sh, tv);
        double ts = 0.0, tt = 0.0;
        KRY_CHECK(K.dot(tv, sv, &ts));
        KRY_CHECK(K.dot(tv, tv, &tt));
        omega = ts / tt;
        K.axpy(alpha, ph, x);
        K.axpy(omega, sh, x);
        K.lin2(1.0, sv, -omega, tv, r);
        rho = rho_new;
        KRY_CHECK(K.norm(r, rn));
        if (!(*rn > target)) break;
    }
    *its = it;
    return SIL_OK;
}

sil_status run_gcr(Krylov& K, int m, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    KRY_CHECK(K.alloc(2 * m + 1));
    double* r = K.vec(2 * m);
    K.copy(b, r);
    KRY_CHECK(K.norm(b, rn));
    int it = 0, k = 0;
    while (it < max_iter) {
        if (k == m) k = 0;
        double *P = K.vec(k), *Q = K.vec(m + k);
        K.precond(r, P);
        K.spmv(P, Q);
        for (int j = 0; j < k; ++j) {
            double h = 0.0;
            KRY_CHECK(K.dot(Q, K.vec(m + j), &h));
            K.axpy(-h, K.vec(m + j), Q);
            K.axpy(-h, K.vec(j), P);
        }
        double qn = 0.0;
        KRY_CHECK(K.norm(Q, &qn));
        K.divide(Q, qn, Q);
        K.divide(P, qn, P);
        double alpha = 0.0;
        KRY_CHECK(K.dot(r, Q, &alpha));
        K.axpy(alpha, P, x);
        K.axpy(-alpha, Q, r);
        ++k;
        ++it;
        KRY_CHECK(K.norm(r, rn));
        if (!(*rn > target)) break;
    }
    *its = it;
    return SIL_OK;
}

sil_status run_idr(Krylov& K, int s, double const* b, double* x, double target, int max_iter, int* its, double* rn)
{
    int64_t const n = K.n();
    KRY_CHECK(K.alloc(3 * s + 4));
    double *r = K.vec(3 * s), *vv = K.vec(3 * s + 1), *vh = K.vec(3 * s + 2), *tt = K.vec(3 * s + 3);
    auto Pv = [&](int j) { return K.vec(j); };
    auto Gv = [&](int j) { return K.vec(s + j); };
    auto Uv = [&](int j) { return K.vec(2 * s + j); };
    // the shadow space of the CPU restatement: xorshift64 + Box-Muller, the
    // vectors orthonormalised in order (on the host)
    {
        std::vector<std::vector<double>> P(s, std::vector<double>(n));
        uint64_t state = 0x9E3779B97F4A7C15ull;
        auto uniform = [&]() {
            state ^= state << 13;
            state ^= state >> 7;
            state ^= state << 17;
            return (static_cast<double>(state >> 11) + 0.5) / 9007199254740992.0;
        };
        auto hdot = [&](std::vector<double> const& a, std::vector<double> const& c) {
            double t = 0.0;
            for (int64_t i = 0; i < n; ++i) t += a[i] * c[i];
            return t;
        };
        for (int j = 0; j < s; ++j) {
            for (int64_t i = 0; i < n; ++i) {
                double const u1 = uniform(), u2 = uniform();
                P[j][i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
            }
            for (int l = 0; l < j; ++l) {
                double const h = hdot(P[j], P[l]);
                for (int64_t i = 0; i < n; ++i) P[j][i] += -h * P[l][i];
            }
            double const pn = std::sqrt(hdot(P[j], P[j]));
            for (int64_t i = 0; i < n; ++i) P[j][i] /= pn;
            SIL_CUDA_CHECK(cudaMemcpyAsync(Pv(j), P[j].data(), n * sizeof(double), cudaMemcpyHostToDevice, K.stream()));
        }
        SIL_CUDA_CHECK(cudaStreamSynchronize(K.stream()));
    }
    std::vector<double> Mm(static_cast<size_t>(s) * s, 0.0), f(s), c(s);
    for (int j = 0; j < s; ++j) Mm[j * s + j] = 1.0;
    K.copy(b, r);
    double om = 1.0;
    KRY_CHECK(K.norm(b, rn));
    int it = 0;
    while (it < max_iter) {
        for (int j = 0; j < s; ++j) KRY_CHECK(K.dot(Pv(j), r, &f[j]));
        for (int k = 0; k < s && it < max_iter; ++k) {
            for (int i = k; i < s; ++i) {
                double acc = f[i];
                for (int j = k; j < i; ++j) acc -= Mm[i * s + j] * c[j];
                c[i] = acc / Mm[i * s + i];
            }
            K.copy(r, vv);
            for (int i = k; i < s; ++i) K.axpy(-c[i], Gv(i), vv);
            K.precond(vv, vh);
            // U_k = om vh + sum_{j >= k} c_j U_j (U_k's old value included)
            K.lin2(om, vh, c[k], Uv(k), Uv(k));
            for (int j = k + 1; j < s; ++j) K.axpy(c[j], Uv(j), Uv(k));
            K.spmv(Uv(k), Gv(k));
            for (int i = 0; i < k; ++i) {
                double pg = 0.0;
                KRY_CHECK(K.dot(Pv(i), Gv(k), &pg));
                double const a = pg / Mm[i * s + i];
                K.axpy(-a, Gv(i), Gv(k));
                K.axpy(-a, Uv(i), Uv(k));
            }
            for (int i = k; i < s; ++i) KRY_CHECK(K.dot(Pv(i), Gv(k), &Mm[i * s + k]));
            double const beta = f[k] / Mm[k * s + k];
            K.axpy(-beta, Gv(k), r);
            K.axpy(beta, Uv(k), x);
            ++it;
            KRY_CHECK(K.norm(r, rn));
            if (!(*rn > target)) break;
            for (int i = k + 1; i < s; ++i) f[i] -= beta * Mm[i * s + k];
        }
        if (!(*rn > target) || it >= max_iter) break;
        K.precond(r, vh);
        K.spmv(vh, tt);
        double tn = 0.0, tr = 0.0, rr = 0.0;
        KRY_CHECK(K.dot(tt, tt, &tn));
        KRY_CHECK(K.dot(tt, r, &tr));
        KRY_CHECK(K.norm(r, &rr));
        om = tr / tn;
        double const rho = std::fabs(tr) / (std::sqrt(tn) * rr);
        if (rho < 0.7) om *= 0.7 / rho;
        K.axpy(-om, tt, r);
        K.axpy(om, vh, x);
        ++it;
        KRY_CHECK(K.norm(r, rn));
        if (!(*rn > target)) break;
    }
    *its = it;
    return SIL_OK;
}

#undef KRY_CHECK

}  // namespace
}  // namespace sil

using namespace sil;

extern "C" {

sil_status sil_mag2d_assemble(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu, sil_csr* out)
{
    if (out == nullptr || node_mu == nullptr) return fail(SIL_ERR_INVALID, "sil_mag2d_assemble: NULL argument");
    *out = nullptr;
    if (nx < 3 || ny < 3) return fail(SIL_ERR_INVALID, "sil_mag2d_assemble: need at least 3x3 nodes");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    Probe const g {2, static_cast<int>(nx), static_cast<int>(ny), 1};
    return assemble(s, g, nx * ny, 9,
                    [&](double const* v, double* y) { return sil_mag2d_apply(stream, nx, ny, node_mu, v, y); }, out);
}

sil_status sil_mag3d_assemble(sil_stream stream, const sil_mag3d_problem* problem, sil_csr* out)
{
    if (out == nullptr || problem == nullptr) return fail(SIL_ERR_INVALID, "sil_mag3d_assemble: NULL argument");
    *out = nullptr;
    sil_mag3d_problem const& q = *problem;
    if (q.nx < 3 || q.ny < 3 || q.nz < 3) return fail(SIL_ERR_INVALID, "sil_mag3d_assemble: need at least 3x3x3 nodes");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    Probe const g {3, static_cast<int>(q.nx), static_cast<int>(q.ny), static_cast<int>(q.nz)};
    return assemble(s, g, 3 * q.nx * q.ny * q.nz, 81,
                    [&](double const* v, double* y) { return sil_mag3d_apply(stream, problem, v, y); }, out);
}

sil_status sil_mag2d_nl_assemble_jacobian(sil_stream stream, const sil_mag2d_nl_problem* problem,
                                          const double* state, sil_csr* out)
{
    if (out == nullptr || problem == nullptr || state == nullptr)
        return fail(SIL_ERR_INVALID, "sil_mag2d_nl_assemble_jacobian: NULL argument");
    *out = nullptr;
    sil_mag2d_nl_problem const& q = *problem;
    if (q.nx < 3 || q.ny < 3) return fail(SIL_ERR_INVALID, "sil_mag2d_nl_assemble_jacobian: need at least 3x3 nodes");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    Probe const g {2, static_cast<int>(q.nx), static_cast<int>(q.ny), 1};
    return assemble(s, g, q.nx * q.ny, 9,
                    [&](double const* v, double* y) { return sil_mag2d_nl_apply_jacobian(stream, problem, state, v, y); },
                    out);
}

sil_status sil_mag3d_nl_assemble_jacobian(sil_stream stream, const sil_mag3d_nl_problem* problem,
                                          const double* state, sil_csr* out)
{
    if (out == nullptr || problem == nullptr || state == nullptr)
        return fail(SIL_ERR_INVALID, "sil_mag3d_nl_assemble_jacobian: NULL argument");
    *out = nullptr;
    sil_mag3d_nl_problem const& q = *problem;
    if (q.nx < 3 || q.ny < 3 || q.nz < 3)
        return fail(SIL_ERR_INVALID, "sil_mag3d_nl_assemble_jacobian: need at least 3x3x3 nodes");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    Probe const g {3, static_cast<int>(q.nx), static_cast<int>(q.ny), static_cast<int>(q.nz)};
    return assemble(s, g, 3 * q.nx * q.ny * q.nz, 81,
                    [&](double const* v, double* y) { return sil_mag3d_nl_apply_jacobian(stream, problem, state, v, y); },
                    out);
}

sil_status sil_csr_get(sil_csr m, int64_t* n, int64_t* nnz, const int32_t** row_ptr, const int32_t** col,
                       const double** val)
{
    if (m == nullptr) return fail(SIL_ERR_INVALID, "sil_csr_get: NULL matrix");
    if (n != nullptr) *n = m->n;
    if (nnz != nullptr) *nnz = m->nnz;
    if (row_ptr != nullptr) *row_ptr = m->ptr;
    if (col != nullptr) *col = m->col;
    if (val != nullptr) *val = m->val;
    return SIL_OK;
}

sil_status sil_csr_copy(sil_stream stream, sil_csr m, int32_t* row_ptr, int32_t* col, double* val)
{
    if (m == nullptr || row_ptr == nullptr || col == nullptr || val == nullptr)
        return fail(SIL_ERR_INVALID, "sil_csr_copy: NULL argument");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    SIL_CUDA_CHECK(cudaMemcpyAsync(row_ptr, m->ptr, (m->n + 1) * sizeof(int32_t), cudaMemcpyDefault, s));
    if (m->nnz > 0) {
        SIL_CUDA_CHECK(cudaMemcpyAsync(col, m->col, m->nnz * sizeof(int32_t), cudaMemcpyDefault, s));
        SIL_CUDA_CHECK(cudaMemcpyAsync(val, m->val, m->nnz * sizeof(double), cudaMemcpyDefault, s));
    }
    SIL_CUDA_CHECK(cudaStreamSynchronize(s));
    return SIL_OK;
}

sil_status sil_csr_spmv(sil_stream stream, sil_csr m, const double* x, double* y)
{
    if (m == nullptr || x == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_csr_spmv: NULL argument");
    spmv_kernel<<<grid_of(m->n), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(m->n, m->ptr, m->col, m->val, x, y);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

void sil_csr_destroy(sil_csr m) { delete m; }

sil_status sil_csr_precond_create(sil_stream stream, sil_csr m, const sil_menu_settings* settings,
                                  sil_csr_precond* out)
{
    if (m == nullptr || settings == nullptr || out == nullptr)
        return fail(SIL_ERR_INVALID, "sil_csr_precond_create: NULL argument");
    *out = nullptr;
    if (settings->kind < SIL_PC_IDENTITY || settings->kind > SIL_PC_GENERAL_ISAI)
        return fail(SIL_ERR_INVALID, "sil_csr_precond_create: unknown preconditioner kind");
    sil_menu_settings const cfg = with_defaults(*settings);
    if (!(cfg.chebyshev_upper_bound > cfg.chebyshev_lower_bound))
        return fail(SIL_ERR_INVALID, "sil_csr_precond_create: Chebyshev bounds must satisfy lower < upper");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    auto P = std::make_unique<sil_csr_precond_s>();
    P->A = m;
    P->cfg = cfg;
    int64_t const n = m->n;
    P->n = n;
    unsigned const G = grid_of(n);
    SIL_CUDA_CHECK(cudaMalloc(&P->diag, std::max<int64_t>(1, n) * sizeof(double)));
    SIL_CUDA_CHECK(cudaMalloc(&P->dinv, std::max<int64_t>(1, n) * sizeof(double)));
    SIL_CUDA_CHECK(cudaMalloc(&P->scratch, std::max<int64_t>(1, 3 * n) * sizeof(double)));
    diag_kernel<<<G, kBlock, 0, s>>>(n, m->ptr, m->col, m->val, P->diag, P->dinv);
    SIL_CUDA_CHECK(cudaGetLastError());
    int const kind = cfg.kind;
    if (kind == SIL_PC_SPD_ISAI || kind == SIL_PC_GENERAL_ISAI || kind == SIL_PC_SSOR ||
        kind == SIL_PC_SYMMETRIC_GAUSS_SEIDEL) {
        // the sparsity pattern on the host (setup)
        std::vector<int32_t> hptr(n + 1), hcol(m->nnz);
        SIL_CUDA_CHECK(cudaMemcpyAsync(hptr.data(), m->ptr, (n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        if (m->nnz > 0)
            SIL_CUDA_CHECK(cudaMemcpyAsync(hcol.data(), m->col, m->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        SIL_CUDA_CHECK(cudaStreamSynchronize(s));
        if (kind == SIL_PC_SSOR || kind == SIL_PC_SYMMETRIC_GAUSS_SEIDEL) {
            std::vector<int32_t> rows;
            levels(hptr, hcol, true, rows, P->fwd_lev);
            if (sil_status st = upload(&P->fwd_rows, rows, s); st != SIL_OK) return st;
            levels(hptr, hcol, false, rows, P->bwd_lev);
            if (sil_status st = upload(&P->bwd_rows, rows, s); st != SIL_OK) return st;
            // single-launch sweeps (int row offsets)
            if (n > 0 && n < (int64_t(1) << 31)) {
                if (sil_status st = upload(&P->fwd_lev_d, P->fwd_lev, s); st != SIL_OK) return st;
                if (sil_status st = upload(&P->bwd_lev_d, P->bwd_lev, s); st != SIL_OK) return st;
            }
        } else {
            bool const spd = kind == SIL_PC_SPD_ISAI;
            std::vector<int32_t> mp(n + 1, 0), mc;
            for (int64_t i = 0; i < n; ++i) {
                for (int32_t k = hptr[i]; k < hptr[i + 1]; ++k)
                    if (!spd || hcol[k] <= i) mc.push_back(hcol[k]);
                mp[i + 1] = static_cast<int32_t>(mc.size());
            }
            if (sil_status st = upload(&P->mptr, mp, s); st != SIL_OK) return st;
            if (sil_status st = upload(&P->mcol, mc, s); st != SIL_OK) return st;
            SIL_CUDA_CHECK(cudaMalloc(&P->mval, std::max<size_t>(1, mc.size()) * sizeof(double)));
            int* bad = nullptr;
            SIL_CUDA_CHECK(cudaMalloc(&bad, sizeof(int)));
            SIL_CUDA_CHECK(cudaMemsetAsync(bad, 0, sizeof(int), s));
            isai_kernel<<<G, kBlock, 0, s>>>(n, spd ? 1 : 0, m->ptr, m->col, m->val, P->mptr, P->mcol, P->mval, bad);
            int hbad = 0;
            cudaError_t const e1 = cudaGetLastError();
            cudaError_t const e2 = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
            cudaError_t const e3 = cudaStreamSynchronize(s);
            cudaFree(bad);
            SIL_CUDA_CHECK(e1);
            SIL_CUDA_CHECK(e2);
            SIL_CUDA_CHECK(e3);
            if (hbad) return fail(SIL_ERR_INVALID, "sil_csr_precond_create: singular ISAI system or a row longer than 32");
            if (spd) {
                // Z^T: rows = columns of Z, entries in ascending row of Z
                std::vector<int32_t> tp(n + 1, 0), tc(mc.size()), perm(mc.size());
                for (int32_t c : mc) ++tp[c + 1];
                for (int64_t i = 0; i < n; ++i) tp[i + 1] += tp[i];
                std::vector<int32_t> fill(tp.begin(), tp.end() - 1);
                for (int64_t i = 0; i < n; ++i)
                    for (int32_t e = mp[i]; e < mp[i + 1]; ++e) {
                        int32_t const pos = fill[mc[e]]++;
                        tc[pos] = static_cast<int32_t>(i);
                        perm[e] = pos;
                    }
                int32_t* dperm = nullptr;
                if (sil_status st = upload(&P->tptr, tp, s); st != SIL_OK) return st;
                if (sil_status st = upload(&P->tcol, tc, s); st != SIL_OK) return st;
                SIL_CUDA_CHECK(cudaMalloc(&P->tval, std::max<size_t>(1, mc.size()) * sizeof(double)));
                if (sil_status st = upload(&dperm, perm, s); st != SIL_OK) return st;
                gather_kernel<<<grid_of(static_cast<int64_t>(mc.size())), kBlock, 0, s>>>(
                        static_cast<int64_t>(mc.size()), dperm, P->mval, P->tval);
                cudaError_t const e4 = cudaGetLastError();
                cudaError_t const e5 = cudaStreamSynchronize(s);
                cudaFree(dperm);
                SIL_CUDA_CHECK(e4);
                SIL_CUDA_CHECK(e5);
            }
        }
    }
    SIL_CUDA_CHECK(cudaStreamSynchronize(s));
    *out = P.release();
    return SIL_OK;
}

sil_status sil_csr_precond_apply(sil_stream stream, sil_csr_precond p, const double* r, double* z)
{
    if (p == nullptr || r == nullptr || z == nullptr) return fail(SIL_ERR_INVALID, "sil_csr_precond_apply: NULL argument");
    precond_launch(*p, static_cast<cudaStream_t>(stream), r, z, nullptr);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

void sil_csr_precond_destroy(sil_csr_precond p) { delete p; }

sil_status sil_csr_solve(sil_stream stream, sil_csr m, sil_csr_precond pc, const double* rhs, double* x,
                         const sil_solve_settings* settings, sil_solve_diagnostics* diag)
{
    if (m == nullptr || pc == nullptr || rhs == nullptr || x == nullptr || settings == nullptr || diag == nullptr)
        return fail(SIL_ERR_INVALID, "sil_csr_solve: NULL argument");
    if (pc->A != m) return fail(SIL_ERR_INVALID, "sil_csr_solve: preconditioner built for another matrix");
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    double const tol = settings->relative_tolerance > 0 ? settings->relative_tolerance : 1e-10;
    int const max_iter = settings->max_iterations > 0 ? settings->max_iterations : 100000;
    int64_t const n = m->n;
    unsigned const G = grid_of(n);
    DevBuf buf;
    size_t const vb = (static_cast<size_t>(n) * sizeof(double) + 255) / 256 * 256;
    size_t const pb = (static_cast<size_t>(G) * sizeof(double) + 255) / 256 * 256;
    SIL_CUDA_CHECK(cudaMalloc(&buf.p, 4 * vb + pb + 256));
    char* base = static_cast<char*>(buf.p);
    double *r = reinterpret_cast<double*>(base), *z = reinterpret_cast<double*>(base + vb),
           *p = reinterpret_cast<double*>(base + 2 * vb), *q = reinterpret_cast<double*>(base + 3 * vb);
    double* part = reinterpret_cast<double*>(base + 4 * vb);
    CgState* st = reinterpret_cast<CgState*>(base + 4 * vb + pb);
    int const np = static_cast<int>(G);
    cg_start_kernel<<<G, kBlock, 0, s>>>(n, rhs, x, r, part);
    cg_init_kernel<<<1, kBlock, 0, s>>>(part, np, st, max_iter);
    precond_launch(*pc, s, r, z, st);
    dot_kernel<<<G, kBlock, 0, s>>>(n, r, z, part, st);
    cg_rz_kernel<<<1, kBlock, 0, s>>>(part, np, st);
    cg_direction_kernel<<<G, kBlock, 0, s>>>(n, part, np, z, p, st, 1);
    SIL_CUDA_CHECK(cudaGetLastError());
    // A chunk of iterations captured once as a CUDA graph (every kernel does
    // nothing once the state is done) and replayed until convergence, the
    // state read back after each replay.  SSOR / symmetric Gauss-Seidel run
    // each triangular sweep as one launch; where they fall back to one
    // launch per level (2^31 rows or more), the chunks are shorter (at most
    // about 4,096 launches per graph).
    int const per_apply = pc->fwd_lev_d != nullptr ? 10 : static_cast<int>(pc->fwd_lev.size() + pc->bwd_lev.size()) + 8;
    int const chunk = std::max(1, std::min(16, 4096 / per_apply));
    auto issue = [&](cudaStream_t cs) {
        for (int c = 0; c < chunk; ++c) {
            cg_spmv_kernel<<<G, kBlock, 0, cs>>>(n, m->ptr, m->col, m->val, p, q, part, st);
            cg_alpha_kernel<<<1, kBlock, 0, cs>>>(part, np, st);
            cg_update_kernel<<<G, kBlock, 0, cs>>>(n, x, r, p, q, part, st);
            cg_check_kernel<<<1, kBlock, 0, cs>>>(part, np, st, tol, max_iter);
            precond_launch(*pc, cs, r, z, st);
            dot_kernel<<<G, kBlock, 0, cs>>>(n, r, z, part, st);
            cg_direction_kernel<<<G, kBlock, 0, cs>>>(n, part, np, z, p, st, 0);
            cg_rz_kernel<<<1, kBlock, 0, cs>>>(part, np, st);
        }
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    {
        cudaStream_t cs;
        SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) issue(cs);
        cudaError_t const err2 = cudaStreamEndCapture(cs, &graph);
        if (err == cudaSuccess) err = err2;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
        cudaStreamDestroy(cs);
        if (err != cudaSuccess) {
            if (graph != nullptr) cudaGraphDestroy(graph);
            return cuda_fail(err, "sil_csr_solve: CG graph capture");
        }
    }
    struct GraphGuard
    {
        cudaGraph_t g;
        cudaGraphExec_t e;
        ~GraphGuard()
        {
            cudaGraphExecDestroy(e);
            cudaGraphDestroy(g);
        }
    } guard {graph, exec};
    CgState hs {};
    for (;;) {
        SIL_CUDA_CHECK(cudaGraphLaunch(exec, s));
        SIL_CUDA_CHECK(cudaMemcpyAsync(&hs, st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
        SIL_CUDA_CHECK(cudaStreamSynchronize(s));
        if (hs.done) break;
    }
    *diag = sil_solve_diagnostics {};
    diag->iterations = hs.iters;
    diag->initial_residual_l2 = hs.bn;
    diag->final_residual_l2 = hs.rn;
    diag->final_relative_residual = hs.bn == 0.0 ? 0.0 : hs.rn / hs.bn;
    diag->converged = (hs.bn == 0.0 || hs.rn <= tol * hs.bn) ? 1 : 0;
    diag->status = std::isfinite(hs.rn) ? SIL_OK : SIL_ERR_NONFINITE;
    diag->refinements = 0;
    return SIL_OK;
}

sil_status sil_csr_krylov_solve(sil_stream stream, sil_csr m, sil_csr_precond pc, int32_t solver, int32_t dim,
                                const double* rhs, double* x, const sil_solve_settings* settings,
                                sil_solve_diagnostics* diag)
{
    if (m == nullptr || pc == nullptr || rhs == nullptr || x == nullptr || settings == nullptr || diag == nullptr)
        return fail(SIL_ERR_INVALID, "sil_csr_krylov_solve: NULL argument");
    if (pc->A != m) return fail(SIL_ERR_INVALID, "sil_csr_krylov_solve: preconditioner built for another matrix");
    if (solver < SIL_KRYLOV_CG || solver > SIL_KRYLOV_IDR)
        return fail(SIL_ERR_INVALID, "sil_csr_krylov_solve: unknown solver");
    if (dim < 0) return fail(SIL_ERR_INVALID, "sil_csr_krylov_solve: negative Krylov dimension");
    if (solver == SIL_KRYLOV_CG) return sil_csr_solve(stream, m, pc, rhs, x, settings, diag);
    cudaStream_t const s = static_cast<cudaStream_t>(stream);
    double const tol = settings->relative_tolerance > 0 ? settings->relative_tolerance : 1e-10;
    int const max_iter = settings->max_iterations > 0 ? settings->max_iterations : 100000;
    SIL_CUDA_CHECK(cudaMemsetAsync(x, 0, static_cast<size_t>(m->n) * sizeof(double), s));
    Krylov K(s, *m, *pc);
    double bn = 0.0;
    {
        Krylov N(s, *m, *pc);
        if (sil_status st = N.alloc(0); st != SIL_OK) return st;
        if (sil_status st = N.norm(rhs, &bn); st != SIL_OK) return st;
    }
    *diag = sil_solve_diagnostics {};
    diag->initial_residual_l2 = bn;
    int its = 0;
    double rn = bn;
    if (bn > 0.0) {
        double const target = tol * bn;
        int const d = dim > 0 ? dim : (solver == SIL_KRYLOV_IDR ? 8 : 100);
        sil_status st = SIL_OK;
        switch (solver) {
        case SIL_KRYLOV_MINRES: st = run_minres(K, rhs, x, target, max_iter, &its, &rn); break;
        case SIL_KRYLOV_FCG: st = run_fcg(K, rhs, x, target, max_iter, &its, &rn); break;
        case SIL_KRYLOV_GMRES: st = run_gmres(K, d, rhs, x, target, max_iter, &its, &rn); break;
        case SIL_KRYLOV_BICGSTAB: st = run_bicgstab(K, rhs, x, target, max_iter, &its, &rn); break;
        case SIL_KRYLOV_GCR: st = run_gcr(K, d, rhs, x, target, max_iter, &its, &rn); break;
        default: st = run_idr(K, d, rhs, x, target, max_iter, &its, &rn); break;
        }
        if (st != SIL_OK) return st;
        SIL_CUDA_CHECK(cudaGetLastError());
    }
    SIL_CUDA_CHECK(cudaStreamSynchronize(s));
    diag->iterations = its;
    diag->final_residual_l2 = rn;
    diag->final_relative_residual = bn == 0.0 ? 0.0 : rn / bn;
    diag->converged = (bn == 0.0 || rn <= tol * bn) ? 1 : 0;
    diag->status = std::isfinite(rn) ? SIL_OK : SIL_ERR_NONFINITE;
    return SIL_OK;
}

}  // extern "C"
