// lap2d.cu -- specialised single-pass 2D Hodge Laplacian kernels.
//
//  * 0-form (delta d): one thread per output node, 5-point stencil through
//    L1/L2 (the configuration it serves, 512^2 FP64, is L2 resident).
//  * 1-form (delta d + d delta): persistent column-strip kernel.  Input row
//    tiles of (R rows) x (128 + halo columns) x 2 components are staged into
//    shared memory by TMA (cp.async.bulk.tensor, no multicast) through an
//    S-stage mbarrier ring; each thread owns one output column and marches
//    down the rows keeping a 2-row register window, so every input element
//    leaves HBM once and every output element is written once.
//
// Both kernels evaluate exactly the same expressions, in the same order, as
// the table-driven fused kernel in dec_generic.cu, so the two agree bit for
// bit; both follow the reference composition (laplacian.hpp:27-155,
// codifferential.hpp:439-507) with the Hodge star of an orthogonal grid.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "sil_internal.cuh"

namespace sil {

namespace {

// ------------------------------------------------------------------ 0-form

template <class T>
struct Lap0Params
{
    T const* in;
    T* out;
    int64_t nx, ny;          // input extents (x slow, y fast)
    int64_t in_row;          // input row stride (elements)
    int64_t mx, my;          // output extents
    int64_t out_row;         // output row stride
    int64_t ox, oy;          // output front relative to the input front
    T const* hx;             // padded: [p + 1]
    T const* ihx;
    T const* hy;
    T const* ihy;
};

template <class T>
__global__ void __launch_bounds__(256) lap2d_0form_kernel(Lap0Params<T> P)
{
    int64_t const jj = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    int64_t const ii = blockIdx.y;
    if (jj >= P.my || ii >= P.mx) return;
    int64_t const i = ii + P.ox, j = jj + P.oy;
    auto phi = [&](int64_t p, int64_t q) {
        p = min(max(p, int64_t(0)), P.nx - 1);
        q = min(max(q, int64_t(0)), P.ny - 1);
        return __ldg(P.in + p * P.in_row + q);
    };
    // eta_x(p) = (-hx/hy) * dphi_y(p), eta_y(p) = (hy/hx) * dphi_x(p); zero outside.
    auto eta_x = [&](int64_t p, int64_t q) -> T {
        if (p < 0 || q < 0 || p >= P.nx || q >= P.ny) return T(0);
        T const d = (T(0) - phi(p, q)) + phi(p, q + 1);
        T const f = (T(-1) * __ldg(P.hx + p + 1)) * __ldg(P.ihy + q + 1);
        return f * d;
    };
    auto eta_y = [&](int64_t p, int64_t q) -> T {
        if (p < 0 || q < 0 || p >= P.nx || q >= P.ny) return T(0);
        T const d = (T(0) - phi(p, q)) + phi(p + 1, q);
        T const f = (T(1) * __ldg(P.ihx + p + 1)) * __ldg(P.hy + q + 1);
        return f * d;
    };
    T acc = T(0);
    acc = acc - eta_y(i, j);
    acc = acc + eta_x(i, j);
    acc = acc + eta_y(i - 1, j);
    acc = acc - eta_x(i, j - 1);
    T const dual_codiff = -acc;
    T const f = (T(1) * __ldg(P.ihx + i + 1)) * __ldg(P.ihy + j + 1);
    P.out[ii * P.out_row + jj] = T(-1) * (f * dual_codiff);
}

// ------------------------------------------------------------------ 1-form, TMA

constexpr int kTJ = 128;     // output columns per strip (= threads per CTA)
constexpr int kRows = 8;     // rows per pipeline stage
constexpr int kStages = 4;   // pipeline depth

template <class T>
struct Lap1Traits;
template <>
struct Lap1Traits<double>
{
    static constexpr int kHalo = 1;  // left halo columns in the staged tile
    using Vec = double2;
};
template <>
struct Lap1Traits<float>
{
    static constexpr int kHalo = 2;  // keeps the TMA start 16-byte aligned
    using Vec = float2;
};

template <class T>
__host__ __device__ constexpr int tile_cols()
{
    return kTJ + 2 * Lap1Traits<T>::kHalo;
}

template <class T>
__host__ __device__ constexpr int stage_bytes()
{
    return kRows * tile_cols<T>() * 2 * static_cast<int>(sizeof(T));
}

template <class T>
struct Lap1Params
{
    T* out;
    int64_t out_row;           // output row stride (elements)
    int nx, ny;                // input extents
    int mx, my;                // output extents
    int ox, oy;                // output front relative to the input front
    int strips;                // column strips of width kTJ over the output
    int64_t work;              // strips * mx (strip-major row items)
    T const* hx;               // padded spacing arrays [p + 1]
    T const* ihx;
    T const* hy;
    T const* ihy;
    int* error_flag;           // set when a bounded wait runs out
};

__device__ __forceinline__ uint32_t smem_addr(void const* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false when the bound runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t const addr = smem_addr(bar);
    for (int tries = 0; tries < (1 << 22); ++tries) {
        uint32_t done;
        asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(addr), "r"(parity)
                : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, CUtensorMap const* map, uint64_t* bar, int c0, int c1, int c2)
{
    asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
            ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
            : "memory");
}

template <class T>
__device__ __forceinline__ void issue_stage(CUtensorMap const* map, T* tile, uint64_t* bar, int strip_col0, int row0)
{
    mbar_expect_tx(bar, stage_bytes<T>());
    if constexpr (sizeof(T) == 8) {
        // map dims {2 comps, ny, nx}; tile columns start at strip_col0 - 1
        tma_load_3d(tile, map, bar, 0, strip_col0 - 1, row0);
    } else {
        // map dims {4 (two nodes x 2 comps), ny / 2, nx}; columns start at strip_col0 - 2 (even)
        tma_load_3d(tile, map, bar, 0, (strip_col0 - 2) / 2, row0);
    }
}

template <class T>
__global__ void __launch_bounds__(kTJ) lap2d_1form_tma_kernel(const __grid_constant__ CUtensorMap map, Lap1Params<T> P)
{
    using Vec = typename Lap1Traits<T>::Vec;
    constexpr int H = Lap1Traits<T>::kHalo;
    constexpr int W = tile_cols<T>();
    constexpr int kStageElems = stage_bytes<T>() / static_cast<int>(sizeof(T));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // Stage buffers start on a 128-byte boundary (the launch reserves 128 spare bytes).
    T* tiles = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    __shared__ __align__(8) uint64_t full[kStages];

    int const tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    // Per-slot counts of loads issued and consumed; identical in every thread
    // (all control flow below is block-uniform), only thread 0 issues.
    uint32_t issued[kStages] = {0, 0, 0, 0};
    uint32_t uses[kStages] = {0, 0, 0, 0};
    bool ok = true;

    int64_t const begin = (P.work * blockIdx.x) / gridDim.x;
    int64_t const end = (P.work * (blockIdx.x + 1)) / gridDim.x;
    int64_t item = begin;
    while (item < end && ok) {
        // Segment: one strip, output rows [r_begin, r_end) relative to the output front.
        int const strip = static_cast<int>(item / P.mx);
        int const r_begin = static_cast<int>(item % P.mx);
        int64_t const seg_len = min(end - item, static_cast<int64_t>(P.mx - r_begin));
        int const r_end = r_begin + static_cast<int>(seg_len);
        item += seg_len;

        int const col0 = P.oy + strip * kTJ;  // first output column of the strip (input-relative)
        int const j = col0 + tid;             // this thread's column (input-relative)
        int const i_first = P.ox + r_begin;   // first output row (input-relative)
        int const i_last = P.ox + r_end;      // one past the last output row
        int const load_row0 = i_first - 1;    // input rows [i_first - 1, i_last] are read
        int const nload = i_last - load_row0 + 1;
        int const nstages = (nload + kRows - 1) / kRows;

        // Column spacing factors at q = j-1, j, j+1 (padded arrays, index q + 1;
        // columns past the output are clamped, their results are never stored).
        int const jq = min(j, P.ny - 2);
        T const hy_m = __ldg(P.hy + jq), ihy_m = __ldg(P.ihy + jq);
        T const hy_0 = __ldg(P.hy + jq + 1), ihy_0 = __ldg(P.ihy + jq + 1);
        T const hy_p = __ldg(P.hy + jq + 2), ihy_p = __ldg(P.ihy + jq + 2);
        bool const col_m_in = j - 1 >= 0;
        bool const store_col = j < P.oy + P.my;

        if (tid == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int s = 0; s < kStages && s < nstages; ++s)
                issue_stage<T>(&map, tiles + s * kStageElems, &full[s], col0, load_row0 + s * kRows);
        }
        for (int s = 0; s < kStages && s < nstages; ++s) issued[s] += 1;

        // Window state, all at the previous row r-1 unless noted.
        T a_m = 0, b_m = 0, a_0 = 0, b_0 = 0, a_p = 0;  // components A (x) and B (y) at columns j-1, j, j+1
        T xy_0 = 0, xx_0 = 0, xy_p = 0, xx_p = 0;       // star of the input: xi_y, xi_x at columns j, j+1
        T xy_p_prev = 0;                               // xi_y at row r-2, column j+1
        T eta_prev = 0;                                // eta(r-2, j)
        T delta_prev = 0;                              // delta(r-1, j)
        int r = load_row0;

        for (int st = 0; st < nstages; ++st) {
            int const slot = st % kStages;
            bool const got = mbar_wait(&full[slot], uses[slot] & 1u);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
            T const* tile = tiles + slot * kStageElems;
            int const rows_here = min(kRows, nload - st * kRows);
            for (int rr = 0; rr < rows_here; ++rr, ++r) {
                Vec const* row = reinterpret_cast<Vec const*>(tile + rr * W * 2);
                int const c = tid + H;  // tile column of j
                Vec const vm = row[c - 1], v0 = row[c], vp = row[c + 1];
                T const hx_r = __ldg(P.hx + r + 1), ihx_r = __ldg(P.ihx + r + 1);
                bool const row_in = r >= 0;
                // Star of the 1-form at row r: xi_x = (-hx/hy) B, xi_y = (hy/hx) A, zero outside.
                T const nxx_m = (row_in && col_m_in) ? ((T(-1) * hx_r) * ihy_m) * vm.y : T(0);
                T const nxy_0 = row_in ? ((T(1) * ihx_r) * hy_0) * v0.x : T(0);
                T const nxx_0 = row_in ? ((T(-1) * hx_r) * ihy_0) * v0.y : T(0);
                T const nxy_p = row_in ? ((T(1) * ihx_r) * hy_p) * vp.x : T(0);
                T const nxx_p = row_in ? ((T(-1) * hx_r) * ihy_p) * vp.y : T(0);
                T eta_0 = 0, eta_m = 0, delta_r = 0, delta_up = 0;
                if (r > load_row0) {
                    int const p = r - 1;
                    T const ihx_p = __ldg(P.ihx + p + 1);
                    bool const p_in = p >= 0;
                    // eta = star(d w) at (p, j) and (p, j-1); d sums in chain order.
                    T d0 = T(0);
                    d0 = d0 - b_0;
                    d0 = d0 + a_0;
                    d0 = d0 + v0.y;
                    d0 = d0 - a_p;
                    eta_0 = p_in ? ((T(1) * ihx_p) * ihy_0) * d0 : T(0);
                    T dm = T(0);
                    dm = dm - b_m;
                    dm = dm + a_m;
                    dm = dm + vm.y;
                    dm = dm - a_0;
                    eta_m = (p_in && col_m_in) ? ((T(1) * ihx_p) * ihy_m) * dm : T(0);
                    // delta(r, j): transposed d of xi, star, codifferential sign.
                    T acc = T(0);
                    acc = acc - nxy_0;
                    acc = acc + nxx_0;
                    acc = acc + xy_0;
                    acc = acc - nxx_m;
                    delta_r = T(-1) * (((T(1) * ihx_r) * ihy_0) * (-acc));
                    // delta(r-1, j+1)
                    T acc2 = T(0);
                    acc2 = acc2 - xy_p;
                    acc2 = acc2 + xx_p;
                    acc2 = acc2 + xy_p_prev;
                    acc2 = acc2 - xx_0;
                    delta_up = T(-1) * (((T(1) * ihx_p) * ihy_p) * (-acc2));
                }
                if (r > i_first) {
                    int const i = r - 1;  // output row
                    T const hx_i = __ldg(P.hx + i + 1), ihx_i = __ldg(P.ihx + i + 1);
                    // delta d: transposed d of eta, star, sign -1.
                    T sx = T(0);
                    sx = sx - eta_0;
                    sx = sx + eta_prev;
                    T sy = T(0);
                    sy = sy - eta_0;
                    sy = sy + eta_m;
                    T const dcx = -sx, dcy = -sy;
                    T const ddx = T(-1) * (((T(-1) * hx_i) * ihy_0) * dcy);
                    T const ddy = T(-1) * (((T(1) * ihx_i) * hy_0) * dcx);
                    // d delta: d of the codifferential.
                    T ex = T(0);
                    ex = ex - delta_prev;
                    ex = ex + delta_r;
                    T ey = T(0);
                    ey = ey - delta_prev;
                    ey = ey + delta_up;
                    if (store_col) {
                        Vec o;
                        o.x = ddx + ex;
                        o.y = ddy + ey;
                        __stcs(reinterpret_cast<Vec*>(P.out + static_cast<int64_t>(i - P.ox) * P.out_row) + (j - P.oy), o);
                    }
                }
                if (r > load_row0) {
                    eta_prev = eta_0;
                    delta_prev = delta_r;
                }
                xy_p_prev = xy_p;
                xy_0 = nxy_0;
                xx_0 = nxx_0;
                xy_p = nxy_p;
                xx_p = nxx_p;
                a_m = vm.x;
                b_m = vm.y;
                a_0 = v0.x;
                b_0 = v0.y;
                a_p = vp.x;
            }
            uses[slot] += 1;
            __syncthreads();  // every thread is done reading this slot
            int const next = st + kStages;
            if (next < nstages) {
                if (tid == 0) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    issue_stage<T>(&map, tiles + slot * kStageElems, &full[slot], col0, load_row0 + next * kRows);
                }
                issued[slot] += 1;
            }
        }
    }
    if (!ok) {
        // Let the copies still in flight land (bounded) before the CTA exits.
        if (tid == 0) {
            for (int s = 0; s < kStages; ++s) {
                while (uses[s] < issued[s]) {
                    mbar_wait(&full[s], uses[s] & 1u);
                    uses[s] += 1;
                }
            }
            atomicExch(P.error_flag, 1);
        }
    }
}

} // namespace

// ------------------------------------------------------------------ host side

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess
            && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <class T>
int lap1_occupancy()
{
    static int blocks = 0;
    if (blocks == 0) {
        int smem = kStages * stage_bytes<T>() + 128;
        cudaFuncSetAttribute(lap2d_1form_tma_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lap2d_1form_tma_kernel<T>, kTJ, smem);
        blocks = b > 0 ? b : 1;
    }
    return blocks;
}

int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

} // namespace

// Fields the specialised 2D kernels accept: both form dims, contiguous DDC
// layout (component fastest, then y, then x), output box inside the input.
bool lap2d_layout_ok(sil_field const& in, sil_field const& out, int ncomp)
{
    if (in.ndims != 2 || out.ndims != 2 || in.ncomp != ncomp || out.ncomp != ncomp) return false;
    if (in.dtype != out.dtype) return false;
    if (ncomp == 2 && (in.comp_stride != 1 || out.comp_stride != 1)) return false;
    if (in.stride[1] != ncomp || out.stride[1] != ncomp) return false;
    if (in.stride[0] != ncomp * in.extent[1]) return false;
    if (out.stride[0] < ncomp * out.extent[1]) return false;
    for (int d = 0; d < 2; ++d) {
        if (out.front[d] < in.front[d]) return false;
        if (out.front[d] + out.extent[d] > in.front[d] + in.extent[d]) return false;
    }
    return in.extent[0] >= 2 && in.extent[1] >= 2;
}

sil_status launch_lap2d_0form(cudaStream_t stream, Geometry const& geo, sil_field const& in, sil_field const& out)
{
    int64_t const mx = out.extent[0], my = out.extent[1];
    if (mx == 0 || my == 0) return SIL_OK;
    dim3 const block(256);
    dim3 const grid(static_cast<unsigned>((my + 255) / 256), static_cast<unsigned>(mx));
    int64_t const gx = in.front[0] - geo.front[0], gy = in.front[1] - geo.front[1];
    if (in.dtype == SIL_F64) {
        Lap0Params<double> P {static_cast<double const*>(in.data), static_cast<double*>(out.data), in.extent[0],
                              in.extent[1], in.stride[0], mx, my, out.stride[0], out.front[0] - in.front[0],
                              out.front[1] - in.front[1], geo.h[0] + gx, geo.inv_h[0] + gx, geo.h[1] + gy,
                              geo.inv_h[1] + gy};
        lap2d_0form_kernel<double><<<grid, block, 0, stream>>>(P);
    } else {
        Lap0Params<float> P {static_cast<float const*>(in.data), static_cast<float*>(out.data), in.extent[0],
                             in.extent[1], in.stride[0], mx, my, out.stride[0], out.front[0] - in.front[0],
                             out.front[1] - in.front[1], geo.h32[0] + gx, geo.inv_h32[0] + gx, geo.h32[1] + gy,
                             geo.inv_h32[1] + gy};
        lap2d_0form_kernel<float><<<grid, block, 0, stream>>>(P);
    }
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

// The TMA 1-form kernel additionally needs the output box to stay one node
// away from the input's upper edges (no clamped samples), 16-byte aligned
// rows, int-sized extents, and for FP32 an even y extent and even y offset.
bool lap2d_1form_tma_ok(sil_field const& in, sil_field const& out)
{
    if (!lap2d_layout_ok(in, out, 2)) return false;
    int64_t const ox = out.front[0] - in.front[0], oy = out.front[1] - in.front[1];
    if (ox + out.extent[0] > in.extent[0] - 1 || oy + out.extent[1] > in.extent[1] - 1) return false;
    if (in.extent[0] > (1 << 30) || in.extent[1] > (1 << 30)) return false;
    size_t const es = in.dtype == SIL_F64 ? 8 : 4;
    if (reinterpret_cast<uintptr_t>(in.data) % 16 != 0) return false;
    if (reinterpret_cast<uintptr_t>(out.data) % (2 * es) != 0) return false;
    if ((out.stride[0] * es) % (2 * es) != 0) return false;
    if (in.dtype == SIL_F32 && (in.extent[1] % 2 != 0 || oy % 2 != 0)) return false;
    return encode_fn() != nullptr;
}

sil_status launch_lap2d_1form_tma(cudaStream_t stream, Geometry const& geo, sil_field const& in, sil_field const& out,
                                  int* error_flag, int max_ctas)
{
    int64_t const mx = out.extent[0], my = out.extent[1];
    if (mx == 0 || my == 0) return SIL_OK;
    auto encode = encode_fn();
    if (encode == nullptr) return fail(SIL_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
    bool const f64 = in.dtype == SIL_F64;
    CUtensorMap map;
    cuuint64_t dims[3];
    cuuint64_t strides[2];
    cuuint32_t box[3];
    cuuint32_t estr[3] = {1, 1, 1};
    uint64_t const nx = in.extent[0], ny = in.extent[1];
    if (f64) {
        dims[0] = 2;
        dims[1] = ny;
        dims[2] = nx;
        strides[0] = 2 * 8;
        strides[1] = 2 * 8 * ny;
        box[0] = 2;
        box[1] = tile_cols<double>();
        box[2] = kRows;
    } else {
        dims[0] = 4;
        dims[1] = ny / 2;
        dims[2] = nx;
        strides[0] = 4 * 4;
        strides[1] = 2 * 4 * ny;
        box[0] = 4;
        box[1] = tile_cols<float>() / 2;
        box[2] = kRows;
    }
    CUresult const res = encode(&map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                                in.data, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (res != CUDA_SUCCESS) return fail(SIL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    int const strips = static_cast<int>((my + kTJ - 1) / kTJ);
    int64_t const work = static_cast<int64_t>(strips) * mx;
    int64_t const gx = in.front[0] - geo.front[0], gy = in.front[1] - geo.front[1];
    int const resident = sm_count() * (f64 ? lap1_occupancy<double>() : lap1_occupancy<float>());
    int64_t ctas = std::min<int64_t>(work, max_ctas > 0 ? std::min(max_ctas, resident) : resident);
    if (ctas < 1) ctas = 1;
    if (f64) {
        Lap1Params<double> P {static_cast<double*>(out.data), out.stride[0], static_cast<int>(nx), static_cast<int>(ny),
                              static_cast<int>(mx), static_cast<int>(my), static_cast<int>(out.front[0] - in.front[0]),
                              static_cast<int>(out.front[1] - in.front[1]), strips, work, geo.h[0] + gx,
                              geo.inv_h[0] + gx, geo.h[1] + gy, geo.inv_h[1] + gy, error_flag};
        lap2d_1form_tma_kernel<double><<<static_cast<unsigned>(ctas), kTJ, kStages * stage_bytes<double>() + 128, stream>>>(map, P);
    } else {
        Lap1Params<float> P {static_cast<float*>(out.data), out.stride[0], static_cast<int>(nx), static_cast<int>(ny),
                             static_cast<int>(mx), static_cast<int>(my), static_cast<int>(out.front[0] - in.front[0]),
                             static_cast<int>(out.front[1] - in.front[1]), strips, work, geo.h32[0] + gx,
                             geo.inv_h32[0] + gx, geo.h32[1] + gy, geo.inv_h32[1] + gy, error_flag};
        lap2d_1form_tma_kernel<float><<<static_cast<unsigned>(ctas), kTJ, kStages * stage_bytes<float>() + 128, stream>>>(map, P);
    }
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

} // namespace sil
