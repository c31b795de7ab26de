// learned.cu — learned plane proposals that seed patch-match (no reference
// counterpart: the reference seeds every pixel with a 64-plane sweep).
//
//   downsample4_kernel  grey -> quarter-resolution grey (4x4 box mean)
//   costvol_kernel      32-plane fronto-parallel census cost volume at quarter
//                       resolution: integer Hamming sums over a 3x3 window and
//                       K support views, normalised to [0, 1]
//   conv3x3_kernel      3x3 convolution as an implicit GEMM on the 5th-
//                       generation tensor cores (tcgen05.mma, BF16 operands
//                       in shared memory, FP32 accumulator in tensor memory)
//   conv3x3_wgrad_kernel  weight gradient of the same convolution (mma.sync
//                       m16n8k16, BF16 in, FP32 accumulate)
//   loss/Adam kernels   training
// The patch-match init that consumes the predictions (confident pixels take
// the predicted plane, the others fall back to the plane sweep) is
// init_learned_rows_kernel in stereo.cu.
//
// Tensors are NHWC, BF16, channels padded to a multiple of 16.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "rcmvs_internal.cuh"
#include "learned.cuh"

namespace rcmvs {

namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ int find_item(const int32_t* start, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------ downsample
__global__ void downsample4_kernel(const DevView* __restrict__ full, const DevView* __restrict__ quarter,
                                   const int32_t* __restrict__ blk_start, int n_views, const uint8_t* __restrict__ gray,
                                   uint8_t* __restrict__ gray_q) {
    const int v = find_item(blk_start, n_views, blockIdx.x);
    const DevView F = full[v], Q = quarter[v];
    const int64_t i = (int64_t)(blockIdx.x - blk_start[v]) * blockDim.x + threadIdx.x;
    if (i >= (int64_t)Q.w * Q.h) return;
    const int x = (int)(i % Q.w), y = (int)(i / Q.w);
    const uint8_t* g = gray + F.off;
    int s = 0;
#pragma unroll
    for (int dy = 0; dy < 4; ++dy)
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) s += g[(size_t)(4 * y + dy) * F.w + 4 * x + dx];
    gray_q[Q.off + i] = (uint8_t)((s + 8) >> 4);
}

// ------------------------------------------------------------ cost volume
// Output channel p < 32 of a quarter-resolution pixel is the mean Hamming
// fraction of fronto-parallel plane p (inverse depths at the centres of 32
// equal bins of [1/zmax, 1/zmin]) over its clamped 3x3 window and the K
// support views; channel 32 is grey/255; channels 33..47 are zero.
//
// On a fronto-parallel plane every window cell sits at depth d, so the
// count of window cell c -- the Hamming distance between c's census and the
// source census where c's ray at depth d projects -- depends on the cell,
// the plane and the source only, not on which pixel's window holds it.  So
// one block takes a 32x8 tile: per plane, its threads compute each of the
// 34x10 cells (tile + clamped 1-cell halo) once, summed over the sources,
// into shared memory, and every pixel adds its nine cells: the same integer
// sums as evaluating each pixel's window, with 340/256 instead of 9
// projections per pixel and source.  A pixel keeps its 32 costs as packed
// BF16 pairs (in shared memory) and writes its 96-byte record with 16-byte
// stores.
constexpr int CV_TW = 32, CV_TH = 8;
constexpr int CV_HW = CV_TW + 2, CV_HH = CV_TH + 2;

__global__ void __launch_bounds__(CV_TW * CV_TH)
    costvol_kernel(const DevJob* __restrict__ jobs, const int32_t* __restrict__ tile_start, int n_jobs,
                   const int64_t* __restrict__ out_off, const uint64_t* __restrict__ census_q,
                   const float2* __restrict__ rays_q, const uint8_t* __restrict__ gray_q, bf16* __restrict__ out) {
    __shared__ DevSrc s_src[RCMVS_MAX_SOURCES];
    __shared__ uint64_t s_cen[CV_HH * CV_HW];
    __shared__ float2 s_ray[CV_HH * CV_HW];
    __shared__ int s_h[CV_HH * CV_HW];
    __shared__ uint32_t s_out[CV_TW * CV_TH][COSTVOL_PLANES / 2 + 1];  // packed BF16 pairs (+1: no bank conflicts)
    const int j = find_item(tile_start, n_jobs, blockIdx.x);
    const DevJob& J = jobs[j];
    const int t = blockIdx.x - tile_start[j];
    const int tiles_x = (J.w + CV_TW - 1) / CV_TW;
    const int x0 = (t % tiles_x) * CV_TW, y0 = (t / tiles_x) * CV_TH;
    const size_t base = (size_t)J.off;
    const int nsrc = J.nsrc;
    {
        const uint32_t* srcw = reinterpret_cast<const uint32_t*>(J.src);
        uint32_t* dstw = reinterpret_cast<uint32_t*>(s_src);
        for (int i = threadIdx.x; i < nsrc * (int)(sizeof(DevSrc) / 4); i += blockDim.x) dstw[i] = srcw[i];
    }
    for (int c = threadIdx.x; c < CV_HH * CV_HW; c += blockDim.x) {
        const int xx = min(max(x0 - 1 + c % CV_HW, 0), J.w - 1);
        const int yy = min(max(y0 - 1 + c / CV_HW, 0), J.h - 1);
        s_cen[c] = census_q[base + (size_t)yy * J.w + xx];
        s_ray[c] = rays_q[base + (size_t)yy * J.w + xx];
    }
    const int lx = threadIdx.x % CV_TW, ly = threadIdx.x / CV_TW;
    const int x = x0 + lx, y = y0 + ly;
    const bool inside = x < J.w && y < J.h;
    const float norm = 1.0f / (9.0f * 48.0f * (float)max(nsrc, 1));
    uint32_t* packed = s_out[threadIdx.x];
    for (int p = 0; p < COSTVOL_PLANES; ++p) {
        const float inv = J.inv_min + (J.inv_max - J.inv_min) * ((float)p + 0.5f) / (float)COSTVOL_PLANES;
        const float d = 1.0f / inv;
        __syncthreads();  // the staged tile (p = 0) / the previous plane's sums are read
        for (int c = threadIdx.x; c < CV_HH * CV_HW; c += blockDim.x) {
            const float2 r = s_ray[c];
            const uint64_t cref = s_cen[c];
            const float xr = d * r.x, yr = d * r.y;
            int hs = 0;
            for (int s = 0; s < nsrc; ++s) {
                const DevSrc& S = s_src[s];
                const float xs = S.rs[0] * xr + S.rs[1] * yr + S.rs[2] * d + S.ts[0];
                const float ys = S.rs[3] * xr + S.rs[4] * yr + S.rs[5] * d + S.ts[1];
                const float zs = S.rs[6] * xr + S.rs[7] * yr + S.rs[8] * d + S.ts[2];
                int h = 48;
                if (zs >= 1e-3f) {
                    const float xn = __fdividef(xs, zs), yn = __fdividef(ys, zs);
                    const float dist = 1.0f + S.k * (xn * xn + yn * yn);
                    const int u = __float2int_rz(S.f * xn * dist + S.cx);
                    const int v = __float2int_rz(S.f * yn * dist + S.cy);
                    if (u >= 0 && v >= 0 && u < S.w && v < S.h)
                        h = __popcll(cref ^ __ldg(census_q + S.off + (size_t)v * S.w + u));
                }
                hs += h;
            }
            s_h[c] = hs;
        }
        __syncthreads();
        int hsum = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) hsum += s_h[(ly + q / 3) * CV_HW + lx + q % 3];
        const uint32_t b = __bfloat16_as_ushort(__float2bfloat16((float)hsum * norm));
        if (p & 1)
            packed[p >> 1] |= b << 16;
        else
            packed[p >> 1] = b;
    }
    if (!inside) return;
    const int64_t i = (int64_t)y * J.w + x;
    const uint32_t g = __bfloat16_as_ushort(__float2bfloat16((float)gray_q[base + i] * (1.0f / 255.0f)));
    uint4* o = reinterpret_cast<uint4*>(out + (size_t)(out_off[j] + i) * COSTVOL_C);  // 96 B, 16-B aligned
#pragma unroll
    for (int k = 0; k < COSTVOL_PLANES / 8; ++k)
        o[k] = make_uint4(packed[4 * k], packed[4 * k + 1], packed[4 * k + 2], packed[4 * k + 3]);
    o[COSTVOL_PLANES / 8] = make_uint4(g, 0u, 0u, 0u);
    o[COSTVOL_PLANES / 8 + 1] = make_uint4(0u, 0u, 0u, 0u);
}

// ------------------------------------------------------------ convolution
// mma.sync.m16n8k16 BF16 -> FP32.  Fragment layout (PTX ISA, "Matrix
// Fragments for mma.m16n8k16 with floating point type"): lane = 4*g + t;
// A rows g and g+8, columns 2t..2t+1 and 2t+8..2t+9; B column g, rows
// 2t..2t+1 and 2t+8..2t+9; C rows g and g+8, columns 2t..2t+1.
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

constexpr int TILE_H = 8, TILE_W = 16;  // output pixels per block: 8 rows x 16 columns (4 warps x 2 rows)

// ---- 5th-generation tensor cores (tcgen05): the forward/data convolution
// Shared-memory matrix descriptor of a tcgen05.mma operand, no swizzle,
// K-major: 8-row x 16-byte core matrices, `lbo` bytes between core matrices
// adjacent in K, `sbo` bytes between core matrices adjacent in M/N (PTX ISA,
// tcgen05 "Shared memory descriptor"; version 1 at bits 46-47).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of tcgen05.mma.kind::f16: FP32 accumulator (bits
// 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the mbarrier at shared address `bar`; gives
// up after `limit_ns` of wall time (returns false).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

template <int N>
__device__ __forceinline__ void tmem_ld_32x32b(uint32_t taddr, uint32_t* v);
template <>
__device__ __forceinline__ void tmem_ld_32x32b<16>(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
template <>
__device__ __forceinline__ void tmem_ld_32x32b<32>(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}

// Set (never cleared by a kernel) when a tensor-core wait gave up; read and
// cleared by tc_fault_take().
__device__ int g_tc_fault = 0;

constexpr int TC_TW = 8, TC_TH = 16;          // output tile: 16 rows x 8 columns = the 128 rows of M
constexpr int TC_SW = TC_TW + 2;              // staged halo tile width
constexpr int TC_NPIX = (TC_TH + 2) * TC_SW;  // staged pixels
constexpr int TC_GS = 2944;                   // bytes per channel group of a staged tile: 180 x 16, 128-aligned
constexpr int TC_CTAS_PER_SM = 3;
constexpr uint64_t TC_WAIT_NS = 2000000000ull;  // 2 s: far above a tile's few microseconds

template <int CIN, int COUT, bool MASK>
struct ConvSmem {
    static constexpr int KG = CIN / 8;                      // 16-byte channel groups
    static constexpr int STAGES = MASK ? 1 : 2;             // TMA double buffer; thread staging single
    static constexpr int W_BYTES = 9 * KG * COUT * 16;      // weights [tap][group][COUT][8]
    static constexpr int X_BYTES = KG * TC_GS;              // one staged tile [group][pixel][8]
    static constexpr int BYTES = 128 + W_BYTES + STAGES * X_BYTES;  // + alignment slack
    static_assert(W_BYTES % 128 == 0, "128-byte aligned stages");
};

// One channel group of the staged tile by TMA: the box (8 channels, 10
// columns, 18 rows, 1 image) at (c0 = 8 * group, x0 - 1, y0 - 1, n) lands
// as [row][column][8 channels] = [pixel][8 channels], zero filled outside
// the image.  The innermost coordinate is a multiple of 8 elements (16
// bytes); the destination is 128-byte aligned.
__device__ __forceinline__ void tma_load_4d(const void* tmap, uint32_t dst, uint32_t bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];"
        :
        : "r"(dst), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// y = conv3x3(x, w) + b, "same" zero padding; optional ReLU; optional f32
// output.  w: [9][COUT][CIN] BF16.  mask (optional): x is multiplied by
// (mask > 0) on load (ReLU derivative of the layer that produced x).
//
// Implicit GEMM on the tensor cores: D[128 pixels][COUT] = sum over the 9
// taps and CIN/16 channel chunks of A[128 pixels][16 channels] x
// B[16 channels][COUT], one tcgen05.mma (M = 128, N = COUT, K = 16, BF16
// operands in shared memory, FP32 accumulator in tensor memory) per tap and
// chunk, issued by one thread.  The output tile is 16 rows x 8 columns, so
// every 8 consecutive rows of A are 8 consecutive pixels of one staged row:
// staging the halo tile as [channel group of 8][pixel][8 channels] makes
// every tap's A a canonical K-major operand in place (core matrix = 8
// pixels x 16 bytes; the next 8 rows of A are the next staged row, 10 pixels
// on; the next 8 channels are the next channel group), so no im2col copy is
// made.  The weights are staged once per CTA as [tap][channel group][COUT][8
// channels].  Persistent CTAs loop over the tiles.  Without a mask the tile
// arrives by TMA (one box per channel group, zero fill at the borders) into
// a double buffer: thread 0 starts the next tile's loads before the current
// tile's MMAs, so they overlap the MMAs and the epilogue.  With a mask (the
// backward pass) the threads stage the tile, masked, into one buffer.  The
// accumulator (COUT f32 columns of 128 lanes) is read back by the four warps
// with tcgen05.ld (warp w owns lanes 32w..32w+31).  Every wait is bounded:
// on a time-out the CTA flags g_tc_fault, waits once more for what it has in
// flight, frees its tensor memory and returns.
template <int CIN, int COUT, bool RELU, bool OUT_F32, bool MASK>
__global__ void __launch_bounds__(128) conv3x3_kernel(const __grid_constant__ CUtensorMap tmap,
                                                      const bf16* __restrict__ x, const bf16* __restrict__ mask, int N,
                                                      int H, int W, const bf16* __restrict__ wgt,
                                                      const float* __restrict__ bias, void* __restrict__ y) {
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "conv3x3 shape");
    using L = ConvSmem<CIN, COUT, MASK>;
    constexpr int KG = L::KG;
    constexpr bool TMA = !MASK;
    constexpr uint32_t IDESC = umma_idesc_bf16(128, COUT);
    constexpr uint32_t TILE_TX = (uint32_t)KG * TC_NPIX * 16;  // bytes one tile's boxes deliver
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[3];  // [0], [1]: tile loaded (per stage); [2]: MMAs done
    __shared__ uint32_t s_taddr;
    __shared__ float s_bias[COUT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // 128-byte aligned base (TMA destinations)
    const uint32_t raw_a = smem_u32(smem);
    const uint32_t base_a = (raw_a + 127u) & ~127u;
    unsigned char* base = smem + (base_a - raw_a);
    uint4* sw = reinterpret_cast<uint4*>(base);
    const uint32_t sw_a = base_a, sx_a0 = base_a + L::W_BYTES;
    const uint32_t full0 = smem_u32(&bars[0]), full1 = smem_u32(&bars[1]);
    const uint32_t mma_a = smem_u32(&bars[2]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(32));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(full0, 1);
        mbar_init(full1, 1);
        mbar_init(mma_a, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 9 * KG * COUT; i += 128) {
        const int co = i % COUT, g = (i / COUT) % KG, tap = i / (COUT * KG);
        sw[i] = *reinterpret_cast<const uint4*>(wgt + (size_t)(tap * COUT + co) * CIN + g * 8);
    }
    if (tid < COUT) s_bias[tid] = bias ? bias[tid] : 0.f;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;
    const int tiles_x = (W + TC_TW - 1) / TC_TW, tiles_y = (H + TC_TH - 1) / TC_TH;
    const int per_img = tiles_x * tiles_y, tiles = per_img * N;
    auto load_tile = [&](int t, int s) {  // thread 0: the TMA boxes of tile t into stage s
        const int n = t / per_img, r = t % per_img;
        const int y0 = (r / tiles_x) * TC_TH, x0 = (r % tiles_x) * TC_TW;
        const uint32_t bar = s ? full1 : full0;
        mbar_expect_tx(bar, TILE_TX);
#pragma unroll
        for (int g = 0; g < KG; ++g)
            tma_load_4d(&tmap, sx_a0 + (uint32_t)(s * L::X_BYTES + g * TC_GS), bar, 8 * g, x0 - 1, y0 - 1, n);
    };
    // loads issued into and waited for per stage (the same in every thread)
    uint32_t issued0 = 0, issued1 = 0, landed0 = 0, landed1 = 0;
    uint32_t mma_issued = 0, mma_done = 0;
    bool ok = true;
    if (TMA && (int)blockIdx.x < tiles) {
        if (tid == 0) load_tile(blockIdx.x, 0);
        issued0 = 1;
    }
    int it = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
        const int s = TMA ? (it & 1) : 0;
        const int n = t / per_img, r = t % per_img;
        const int y0 = (r / tiles_x) * TC_TH, x0 = (r % tiles_x) * TC_TW;
        const size_t img = (size_t)n * H * W;
        if (TMA) {
            // the other stage was read by the previous tile's MMAs, which completed
            if (t + (int)gridDim.x < tiles) {
                if (tid == 0) load_tile(t + gridDim.x, s ^ 1);
                if (s) ++issued0; else ++issued1;
            }
            const bool got = mbar_wait(s ? full1 : full0, (s ? landed1 : landed0) & 1u, TC_WAIT_NS);
            if (!__syncthreads_and(got)) {
                ok = false;
                break;
            }
            if (s) ++landed1; else ++landed0;
        } else {
            uint4* sx = reinterpret_cast<uint4*>(base + L::W_BYTES);
            for (int i = tid; i < TC_NPIX * KG; i += 128) {
                const int g = i % KG, p = i / KG;
                const int gy = y0 - 1 + p / TC_SW, gx = x0 - 1 + p % TC_SW;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
                    const size_t gi = (img + (size_t)gy * W + gx) * CIN + g * 8;
                    v = *reinterpret_cast<const uint4*>(x + gi);
                    if (MASK) {
                        const uint4 m = *reinterpret_cast<const uint4*>(mask + gi);
                        const bf16* mv = reinterpret_cast<const bf16*>(&m);
                        bf16* xv = reinterpret_cast<bf16*>(&v);
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            if (!(__bfloat162float(mv[q]) > 0.0f)) xv[q] = __float2bfloat16(0.0f);
                    }
                }
                sx[g * (TC_GS / 16) + p] = v;
            }
            // generic-proxy smem writes -> visible to the tensor core (async proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint32_t sx_a = sx_a0 + (uint32_t)(s * L::X_BYTES);
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                const int ky = tap / 3, kx = tap % 3;
#pragma unroll
                for (int kc = 0; kc < CIN / 16; ++kc) {
                    const uint64_t a =
                        umma_desc(sx_a + (uint32_t)((2 * kc) * TC_GS + (ky * TC_SW + kx) * 16), TC_GS, TC_SW * 16);
                    const uint64_t b = umma_desc(sw_a + (uint32_t)((tap * KG + 2 * kc) * COUT * 16), COUT * 16, 128);
                    umma_bf16(taddr, a, b, IDESC, (tap | kc) != 0 ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mma_a)
                         : "memory");
        }
        ++mma_issued;
        __syncwarp();
        const bool got = mbar_wait(mma_a, mma_done & 1u, TC_WAIT_NS);
        if (!__syncthreads_and(got)) {
            ok = false;
            break;
        }
        ++mma_done;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t v[COUT];
        tmem_ld_32x32b<COUT>(taddr + ((uint32_t)(32 * warp) << 16), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int m = 32 * warp + lane, oy = y0 + m / TC_TW, ox = x0 + m % TC_TW;
        if (oy < H && ox < W) {
            const size_t o = (img + (size_t)oy * W + ox) * COUT;
            float f[COUT];
#pragma unroll
            for (int c = 0; c < COUT; ++c) {
                float sv = __uint_as_float(v[c]) + s_bias[c];
                f[c] = RELU ? fmaxf(sv, 0.f) : sv;
            }
            if (OUT_F32) {
                float4* yo = reinterpret_cast<float4*>(reinterpret_cast<float*>(y) + o);
#pragma unroll
                for (int c = 0; c < COUT / 4; ++c) yo[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
            } else {
                uint4* yo = reinterpret_cast<uint4*>(reinterpret_cast<bf16*>(y) + o);
#pragma unroll
                for (int c = 0; c < COUT / 8; ++c)
                    yo[c] = make_uint4(pack2(__float2bfloat16(f[8 * c]), __float2bfloat16(f[8 * c + 1])),
                                       pack2(__float2bfloat16(f[8 * c + 2]), __float2bfloat16(f[8 * c + 3])),
                                       pack2(__float2bfloat16(f[8 * c + 4]), __float2bfloat16(f[8 * c + 5])),
                                       pack2(__float2bfloat16(f[8 * c + 6]), __float2bfloat16(f[8 * c + 7])));
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (!ok) {
        // wait once more for what is still in flight before the smem and the
        // tensor memory are released
        if (tid == 0) atomicExch(&g_tc_fault, 1);
        if (mma_issued > mma_done) mbar_wait(mma_a, mma_done & 1u, TC_WAIT_NS);
        for (uint32_t k = landed0; k < issued0; ++k) mbar_wait(full0, k & 1u, TC_WAIT_NS);
        for (uint32_t k = landed1; k < issued1; ++k) mbar_wait(full1, k & 1u, TC_WAIT_NS);
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(32));
}

// dW[tap][co][ci] += sum_p dy[p][co] * x[p + tap][ci] over the block's pixel
// tiles; dy is masked by (mask > 0) when MASK.  Grid: (tile blocks, 9 taps).
// Per warp: M = COUT rows (co), N = CIN columns (ci), K = 32 of the tile's
// 128 pixels; partial sums are reduced in shared memory and added to dW.
template <int CIN, int COUT, bool MASK>
__global__ void __launch_bounds__(128) conv3x3_wgrad_kernel(const bf16* __restrict__ x, const bf16* __restrict__ dy,
                                                            const bf16* __restrict__ mask, int N, int H, int W,
                                                            float* __restrict__ dW) {
    constexpr int SPX = CIN + 8;
    constexpr int SPY = COUT + 8;
    extern __shared__ __align__(16) unsigned char smem[];
    bf16* sx = reinterpret_cast<bf16*>(smem);
    bf16* sy = sx + (TILE_H + 2) * (TILE_W + 2) * SPX;
    float* red = reinterpret_cast<float*>(sy + TILE_H * TILE_W * SPY);
    const int tap = blockIdx.y, ky = tap / 3, kx = tap % 3;
    const int tiles_x = (W + TILE_W - 1) / TILE_W, tiles_y = (H + TILE_H - 1) / TILE_H;
    const int n_tiles = N * tiles_x * tiles_y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    constexpr int MT = COUT / 16, NT = CIN / 8;
    float acc[MT][NT][4];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[m][nt][0] = acc[m][nt][1] = acc[m][nt][2] = acc[m][nt][3] = 0.f;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int n = tile / (tiles_x * tiles_y), r = tile % (tiles_x * tiles_y);
        const int x0 = (r % tiles_x) * TILE_W, y0 = (r / tiles_x) * TILE_H;
        const size_t img = (size_t)n * H * W;
        __syncthreads();
        for (int i = threadIdx.x; i < (TILE_H + 2) * (TILE_W + 2) * (CIN / 8); i += 128) {
            const int c8 = i % (CIN / 8), p = i / (CIN / 8);
            const int gy = y0 - 1 + p / (TILE_W + 2), gx = x0 - 1 + p % (TILE_W + 2);
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < H && gx >= 0 && gx < W)
                v = *reinterpret_cast<const uint4*>(x + (img + (size_t)gy * W + gx) * CIN + c8 * 8);
            *reinterpret_cast<uint4*>(sx + p * SPX + c8 * 8) = v;
        }
        for (int i = threadIdx.x; i < TILE_H * TILE_W * (COUT / 8); i += 128) {
            const int c8 = i % (COUT / 8), p = i / (COUT / 8);
            const int gy = y0 + p / TILE_W, gx = x0 + p % TILE_W;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy < H && gx < W) {
                const size_t gi = (img + (size_t)gy * W + gx) * COUT + c8 * 8;
                v = *reinterpret_cast<const uint4*>(dy + gi);
                if (MASK) {
                    const uint4 mm = *reinterpret_cast<const uint4*>(mask + gi);
                    const bf16* mv = reinterpret_cast<const bf16*>(&mm);
                    bf16* yv = reinterpret_cast<bf16*>(&v);
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if (!(__bfloat162float(mv[q]) > 0.0f)) yv[q] = __float2bfloat16(0.0f);
                }
            }
            *reinterpret_cast<uint4*>(sy + p * SPY + c8 * 8) = v;
        }
        __syncthreads();
        // warp w: pixels k in [32w, 32w+32) of the tile = 2 k-steps of 16
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int kbase = warp * 32 + ks * 16;
            const int pa = kbase + 2 * t, pb = pa + 8;  // pixel indices of this lane's k pairs
            uint32_t a[MT][4];
#pragma unroll
            for (int m = 0; m < MT; ++m) {
                const int co = m * 16 + g;
                a[m][0] = pack2(sy[pa * SPY + co], sy[(pa + 1) * SPY + co]);
                a[m][1] = pack2(sy[pa * SPY + co + 8], sy[(pa + 1) * SPY + co + 8]);
                a[m][2] = pack2(sy[pb * SPY + co], sy[(pb + 1) * SPY + co]);
                a[m][3] = pack2(sy[pb * SPY + co + 8], sy[(pb + 1) * SPY + co + 8]);
            }
            // x at pixel p shifted by the tap: shared cell (p/16 + ky, p%16 + kx)
            const int xa0 = ((pa / TILE_W) + ky) * (TILE_W + 2) + (pa % TILE_W) + kx;
            const int xa1 = (((pa + 1) / TILE_W) + ky) * (TILE_W + 2) + ((pa + 1) % TILE_W) + kx;
            const int xb0 = ((pb / TILE_W) + ky) * (TILE_W + 2) + (pb % TILE_W) + kx;
            const int xb1 = (((pb + 1) / TILE_W) + ky) * (TILE_W + 2) + ((pb + 1) % TILE_W) + kx;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int ci = nt * 8 + g;
                const uint32_t b0 = pack2(sx[xa0 * SPX + ci], sx[xa1 * SPX + ci]);
                const uint32_t b1 = pack2(sx[xb0 * SPX + ci], sx[xb1 * SPX + ci]);
#pragma unroll
                for (int m = 0; m < MT; ++m) mma_bf16(acc[m][nt], a[m], b0, b1);
            }
        }
    }
    // reduce the 4 warps: red[co][ci]
    __syncthreads();
    for (int i = threadIdx.x; i < COUT * CIN; i += 128) red[i] = 0.f;
    __syncthreads();
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int co = m * 16 + g, ci = nt * 8 + 2 * t;
            atomicAdd(&red[co * CIN + ci], acc[m][nt][0]);
            atomicAdd(&red[co * CIN + ci + 1], acc[m][nt][1]);
            atomicAdd(&red[(co + 8) * CIN + ci], acc[m][nt][2]);
            atomicAdd(&red[(co + 8) * CIN + ci + 1], acc[m][nt][3]);
        }
    __syncthreads();
    for (int i = threadIdx.x; i < COUT * CIN; i += 128) atomicAdd(&dW[(size_t)tap * COUT * CIN + i], red[i]);
}

// db[c] += sum over pixels of dy[p][c] * (mask[p][c] > 0)
template <int C, bool MASK>
__global__ void bias_grad_kernel(const bf16* __restrict__ dy, const bf16* __restrict__ mask, int64_t npx,
                                 float* __restrict__ db) {
    float s[C];
#pragma unroll
    for (int c = 0; c < C; ++c) s[c] = 0.f;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npx; p += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int c = 0; c < C; ++c) {
            float v = __bfloat162float(dy[p * C + c]);
            if (MASK && !(__bfloat162float(mask[p * C + c]) > 0.f)) v = 0.f;
            s[c] += v;
        }
#pragma unroll
    for (int c = 0; c < C; ++c) {
        float v = s[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&db[c], v);
    }
}

// backward-data weights: wt[tap][ci][co] = w[8 - tap][co][ci]
__global__ void flip_weights_kernel(const bf16* __restrict__ w, int cout, int cin, bf16* __restrict__ wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * cout * cin) return;
    const int ci = i % cin, co = (i / cin) % cout, tap = i / (cin * cout);
    wt[((size_t)(8 - tap) * cin + ci) * cout + co] = w[i];
}

__global__ void to_bf16_kernel(const float* __restrict__ a, int64_t n, bf16* __restrict__ b) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

// Loss on the head output (16 channels, f32: t, nx, ny, nz, conf logit, 0...)
// against labels (8 floats: t*, nx*, ny*, nz*, valid, tol, 0, 0):
//   |t - t*| + LN (1 - cos(n, n*)) + LC BCE(sigmoid(c), |t - t*| < tol)
// averaged over valid pixels; writes dL/dout (BF16, 16 channels) and adds the
// summed loss and the valid count to acc[0..1].
constexpr float LN = 1.0f, LC = 0.1f;
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ lab, int64_t npx, float inv_n,
                            bf16* __restrict__ dout, float* __restrict__ acc) {
    float l = 0.f, cnt = 0.f;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npx; p += (int64_t)gridDim.x * blockDim.x) {
        const float* o = out + p * NET_OUT_C;
        const float* L = lab + p * 8;
        float g[NET_OUT_C];
#pragma unroll
        for (int c = 0; c < NET_OUT_C; ++c) g[c] = 0.f;
        if (L[4] > 0.5f) {
            const float dt = o[0] - L[0];
            l += fabsf(dt);
            g[0] = (dt > 0.f ? 1.f : (dt < 0.f ? -1.f : 0.f));
            const float nl = sqrtf(o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) + 1e-6f;
            const float c = (o[1] * L[1] + o[2] * L[2] + o[3] * L[3]) / nl;
            l += LN * (1.f - c);
#pragma unroll
            for (int a = 0; a < 3; ++a) g[1 + a] = -LN * (L[1 + a] - c * o[1 + a] / nl) / nl;
            const float pr = 1.f / (1.f + __expf(-o[4]));
            const float tgt = fabsf(dt) < L[5] ? 1.f : 0.f;
            l += LC * -(tgt * __logf(fmaxf(pr, 1e-7f)) + (1.f - tgt) * __logf(fmaxf(1.f - pr, 1e-7f)));
            g[4] = LC * (pr - tgt);
            cnt += 1.f;
        }
#pragma unroll
        for (int c = 0; c < NET_OUT_C; ++c) dout[p * NET_OUT_C + c] = __float2bfloat16(g[c] * inv_n);
    }
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_down_sync(0xffffffffu, l, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc, l);
        atomicAdd(acc + 1, cnt);
    }
}

// Adam on the f32 master parameters (gradients scaled by gscale), then the
// BF16 compute copy.  mask[i] = 0 pins padded weights at zero.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m,
                            float* __restrict__ v, const uint8_t* __restrict__ mask, int64_t n, float lr, float b1,
                            float b2, float eps, float bc1, float bc2, float gscale, bf16* __restrict__ pb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!mask[i]) {
        pb[i] = __float2bfloat16(0.f);
        return;
    }
    const float g = gr[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16(pi);
}

}  // namespace

// ------------------------------------------------------------ launchers
cudaError_t launch_downsample4(const DevView* full, const DevView* quarter, const int32_t* blk_start, int n_views,
                               int total_blocks, const uint8_t* gray, uint8_t* gray_q, cudaStream_t st) {
    if (total_blocks <= 0) return cudaSuccess;
    downsample4_kernel<<<total_blocks, 256, 0, st>>>(full, quarter, blk_start, n_views, gray, gray_q);
    return cudaGetLastError();
}

int costvol_tiles(int w, int h) { return ((w + CV_TW - 1) / CV_TW) * ((h + CV_TH - 1) / CV_TH); }

cudaError_t launch_costvol(const DevJob* jobs, const int32_t* blk_start, int n_jobs, int total_blocks,
                           const int64_t* out_off, const uint64_t* census_q, const float2* rays_q,
                           const uint8_t* gray_q, void* out, cudaStream_t st) {
    if (total_blocks <= 0) return cudaSuccess;
    costvol_kernel<<<total_blocks, CV_TW * CV_TH, 0, st>>>(jobs, blk_start, n_jobs, out_off, census_q, rays_q,
                                                           gray_q, reinterpret_cast<bf16*>(out));
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled from the driver, looked up once (no libcuda link).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The NHWC BF16 input as a 4-D tensor (C, W, H, N) for TMA, box (8, 10, 18,
// 1): one channel group of a staged halo tile.
cudaError_t input_tensor_map(const void* x, int cin, int N, int H, int W, CUtensorMap* out) {
    auto enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)cin * 2, (cuuint64_t)W * cin * 2, (cuuint64_t)H * W * cin * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)TC_SW, (cuuint32_t)(TC_TH + 2), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int CIN, int COUT, bool RELU, bool OUT_F32, bool MASK>
static cudaError_t conv_t(const void* x, const void* mask, int N, int H, int W, const void* w, const float* b, void* y,
                          cudaStream_t st) {
    if (N <= 0 || H <= 0 || W <= 0) return cudaSuccess;
    // 16-byte operand loads and stores (and the TMA base address)
    if (((uintptr_t)x | (uintptr_t)w | (uintptr_t)y | (mask ? (uintptr_t)mask : 0)) & 15) return cudaErrorMisalignedAddress;
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    cudaError_t e;
    if (!MASK && (e = input_tensor_map(x, CIN, N, H, W, &tmap))) return e;
    const size_t sm = ConvSmem<CIN, COUT, MASK>::BYTES;
    auto k = conv3x3_kernel<CIN, COUT, RELU, OUT_F32, MASK>;
    if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm))) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
    const long long tiles = (long long)((W + TC_TW - 1) / TC_TW) * ((H + TC_TH - 1) / TC_TH) * N;
    if (tiles > INT_MAX) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(tiles, (long long)sms * TC_CTAS_PER_SM);
    k<<<grid, 128, sm, st>>>(tmap, reinterpret_cast<const bf16*>(x), reinterpret_cast<const bf16*>(mask), N, H, W,
                             reinterpret_cast<const bf16*>(w), b, y);
    return cudaGetLastError();
}

namespace {
__global__ void wait_probe_kernel(uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t bar_a = smem_u32(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool got = mbar_wait(bar_a, 0u, limit_ns);
    if (!__syncthreads_and(got) && threadIdx.x == 0) atomicExch(&g_tc_fault, 1);
}
}  // namespace

cudaError_t launch_wait_probe(uint64_t limit_ns, cudaStream_t st) {
    wait_probe_kernel<<<1, 32, 0, st>>>(limit_ns);
    return cudaGetLastError();
}

int tc_fault_take() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_fault, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_tc_fault, &z, sizeof(int)) != cudaSuccess) return -1;
    }
    return v;
}

cudaError_t launch_conv3x3(int cin, int cout, bool relu, bool out_f32, const void* x, const void* mask, int N, int H,
                           int W, const void* w, const float* b, void* y, cudaStream_t st) {
    const bool m = mask != nullptr;
    if (cin == 48 && cout == 32 && relu && !out_f32 && !m) return conv_t<48, 32, true, false, false>(x, mask, N, H, W, w, b, y, st);
    if (cin == 32 && cout == 32 && relu && !out_f32 && !m) return conv_t<32, 32, true, false, false>(x, mask, N, H, W, w, b, y, st);
    if (cin == 32 && cout == 16 && !relu && out_f32 && !m) return conv_t<32, 16, false, true, false>(x, mask, N, H, W, w, b, y, st);
    // backward data: input = masked upstream gradient, no bias, no ReLU
    if (cin == 16 && cout == 32 && !relu && !out_f32 && !m) return conv_t<16, 32, false, false, false>(x, mask, N, H, W, w, b, y, st);
    if (cin == 32 && cout == 32 && !relu && !out_f32 && m) return conv_t<32, 32, false, false, true>(x, mask, N, H, W, w, b, y, st);
    return cudaErrorInvalidValue;
}

template <int CIN, int COUT, bool MASK>
static cudaError_t wgrad_t(const void* x, const void* dy, const void* mask, int N, int H, int W, float* dW,
                           cudaStream_t st) {
    const size_t sm = sizeof(bf16) * ((TILE_H + 2) * (TILE_W + 2) * (CIN + 8) + TILE_H * TILE_W * (COUT + 8)) +
                      sizeof(float) * COUT * CIN;
    auto k = conv3x3_wgrad_kernel<CIN, COUT, MASK>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e) return e;
    const int tiles = N * ((W + TILE_W - 1) / TILE_W) * ((H + TILE_H - 1) / TILE_H);
    dim3 grid(std::min(tiles, 148 * 2), 9);
    k<<<grid, 128, sm, st>>>(reinterpret_cast<const bf16*>(x), reinterpret_cast<const bf16*>(dy),
                             reinterpret_cast<const bf16*>(mask), N, H, W, dW);
    return cudaGetLastError();
}

cudaError_t launch_conv3x3_wgrad(int cin, int cout, const void* x, const void* dy, const void* mask, int N, int H,
                                 int W, float* dW, cudaStream_t st) {
    const bool m = mask != nullptr;
    if (cin == 48 && cout == 32 && m) return wgrad_t<48, 32, true>(x, dy, mask, N, H, W, dW, st);
    if (cin == 32 && cout == 32 && m) return wgrad_t<32, 32, true>(x, dy, mask, N, H, W, dW, st);
    if (cin == 32 && cout == 16 && !m) return wgrad_t<32, 16, false>(x, dy, mask, N, H, W, dW, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_bias_grad(int c, const void* dy, const void* mask, int64_t npx, float* db, cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>((npx + 255) / 256, 148 * 4);
    if (c == 32 && mask)
        bias_grad_kernel<32, true><<<blocks, 256, 0, st>>>(reinterpret_cast<const bf16*>(dy),
                                                           reinterpret_cast<const bf16*>(mask), npx, db);
    else if (c == 16 && !mask)
        bias_grad_kernel<16, false><<<blocks, 256, 0, st>>>(reinterpret_cast<const bf16*>(dy), nullptr, npx, db);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_flip_weights(const void* w, int cout, int cin, void* wt, cudaStream_t st) {
    const int n = 9 * cout * cin;
    flip_weights_kernel<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const bf16*>(w), cout, cin,
                                                         reinterpret_cast<bf16*>(wt));
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* a, int64_t n, void* b, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    to_bf16_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, n, reinterpret_cast<bf16*>(b));
    return cudaGetLastError();
}

cudaError_t launch_loss(const float* out, const float* lab, int64_t npx, float inv_n, void* dout, float* acc,
                        cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>((npx + 255) / 256, 148 * 4);
    loss_kernel<<<blocks, 256, 0, st>>>(out, lab, npx, inv_n, reinterpret_cast<bf16*>(dout), acc);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, const uint8_t* mask, int64_t n, float lr,
                        float b1, float b2, float eps, float bc1, float bc2, float gscale, void* pb, cudaStream_t st) {
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, g, m, v, mask, n, lr, b1, b2, eps, bc1, bc2, gscale,
                                                             reinterpret_cast<bf16*>(pb));
    return cudaGetLastError();
}

}  // namespace rcmvs
