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
    ~sil_csr_precond_s()
    {
        for (void* p : {static_cast<void*>(diag), static_cast<void*>(dinv), static_cast<void*>(scratch),
                        static_cast<void*>(mptr), static_cast<void*>(mcol), static_cast<void*>(tptr),
                        static_cast<void*>(tcol), static_cast<void*>(mval), static_cast<void*>(tval),
                        static_cast<void*>(fwd_rows), static_cast<void*>(bwd_rows)})
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
    // iterations issued in chunks, the state read back after each chunk
    CgState hs {};
    for (;;) {
        for (int c = 0; c < 16; ++c) {
            cg_spmv_kernel<<<G, kBlock, 0, s>>>(n, m->ptr, m->col, m->val, p, q, part, st);
            cg_alpha_kernel<<<1, kBlock, 0, s>>>(part, np, st);
            cg_update_kernel<<<G, kBlock, 0, s>>>(n, x, r, p, q, part, st);
            cg_check_kernel<<<1, kBlock, 0, s>>>(part, np, st, tol, max_iter);
            precond_launch(*pc, s, r, z, st);
            dot_kernel<<<G, kBlock, 0, s>>>(n, r, z, part, st);
            cg_direction_kernel<<<G, kBlock, 0, s>>>(n, part, np, z, p, st, 0);
            cg_rz_kernel<<<1, kBlock, 0, s>>>(part, np, st);
        }
        SIL_CUDA_CHECK(cudaGetLastError());
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

}  // extern "C"
