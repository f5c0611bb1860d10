// The learned warm start of the pressure solve: a small convolutional network
// that predicts the change of the pressure correction from the same RK stage
// one time step earlier, trained on pairs the solver itself produces.  No
// counterpart in the reference.
//
// Network (fixed): six 3x3 convolutions, 3 -> 32 -> 32 -> 32 -> 32 -> 32 -> 1
// channels, zero padding, ReLU after all but the last; weights held in FP32
// for training and used in BF16 by the forward pass, every product
// accumulated in FP32.  Activations are channel-major planes [C][H][W].
//
// Inputs of a sample (all on the physical cells of the solve range):
//   x0 = rho, x1 = r0 / rms(r0) with r0 = rhs - A phi_prev the residual the
//   previous correction leaves, x2 = phi_prev / rms(phi_prev);
// output y, the predicted change of the correction over rms(phi_prev); the
// warm start takes the Galerkin step along it from phi_prev (k_cnn_apply);
// training target t = (phi - phi_prev) / rms(phi_prev).
//
// Kernels: the four hidden 32 -> 32 layers run on the tensor cores
// (k_conv_umma: tcgen05.mma implicit GEMM, BF16 activations and weights, FP32
// accumulation in tensor memory), forward and input gradient, and their
// weight gradients (k_conv_wgrad_umma, the pixels as the GEMM's K); the first
// (3 -> 32) and last (32 -> 1) layers, too narrow for an MMA tile, are a
// shared-memory tiled direct convolution on the FP32 pipes (one thread per
// pixel, all output channels in registers); the input gradient is the same
// convolution with the taps flipped and the channels swapped, the weight
// gradient per-block partial sums; then the mean-square loss, Adam, and the
// input assembly with the two root mean squares.
#include <cuda_bf16.h>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/pvof.h"
#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

namespace {

constexpr int CNN_TILE = 16;             // output tile edge of a block
constexpr int CNN_HALO = CNN_TILE + 2;   // with the 3x3 halo
constexpr int CNN_CMAX = 32;             // channels of the hidden layers

// forward: out[co][p] = b[co] + sum_ci sum_tap w[co][ci][tap] * in[ci][p + tap]
// (zero outside the H x W plane), then ReLU if relu
template <int COUT>
__global__ void __launch_bounds__(CNN_TILE * CNN_TILE) k_conv3x3(const float *__restrict__ in, int cin,
                                                                 const __nv_bfloat16 *__restrict__ w,
                                                                 const float *__restrict__ b, float *__restrict__ out,
                                                                 int H, int W, int relu)
{
    extern __shared__ float cnn_smem[];
    float (*tile)[CNN_HALO][CNN_HALO] = reinterpret_cast<float (*)[CNN_HALO][CNN_HALO]>(cnn_smem);
    float *ws = cnn_smem + cin * CNN_HALO * CNN_HALO;   // the layer's weights, COUT * cin * 9
    const int tx = threadIdx.x % CNN_TILE, ty = threadIdx.x / CNN_TILE;
    const int i0 = blockIdx.x * CNN_TILE, j0 = blockIdx.y * CNN_TILE;
    const size_t plane = (size_t)H * W;
    for (int q = threadIdx.x; q < cin * CNN_HALO * CNN_HALO; q += blockDim.x) {
        const int c = q / (CNN_HALO * CNN_HALO), r = q % (CNN_HALO * CNN_HALO);
        const int i = i0 + r % CNN_HALO - 1, j = j0 + r / CNN_HALO - 1;
        tile[c][r / CNN_HALO][r % CNN_HALO] = (i >= 0 && i < W && j >= 0 && j < H) ? in[c * plane + (size_t)j * W + i] : 0.0f;
    }
    for (int q = threadIdx.x; q < COUT * cin * 9; q += blockDim.x) ws[q] = __bfloat162float(w[q]);
    __syncthreads();
    const int i = i0 + tx, j = j0 + ty;
    if (i >= W || j >= H) return;
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; co++) acc[co] = b ? b[co] : 0.0f;
    for (int ci = 0; ci < cin; ci++)
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const float x = tile[ci][ty + t / 3][tx + t % 3];
#pragma unroll
            for (int co = 0; co < COUT; co++) acc[co] += x * ws[(co * cin + ci) * 9 + t];
        }
#pragma unroll
    for (int co = 0; co < COUT; co++) {
        float v = acc[co];
        if (relu && v < 0.0f) v = 0.0f;
        out[co * plane + (size_t)j * W + i] = v;
    }
}

// ---------------------------------------------------------------------------
// 32 -> 32 channel 3x3 convolutions on the tensor cores (tcgen05, kind::f16)
// ---------------------------------------------------------------------------
// An implicit GEMM D[p][co] = sum_k A[p][k] B[co][k] over k = tap * 32 + ci
// (288 = 18 MMAs of K = 16): one CTA of 128 threads takes 128 consecutive
// pixels of the flattened H x W plane (the MMA's M = 128, N = 32).  Every
// thread gathers its pixel's im2col row, rounded to BF16, into shared memory,
// the CTA the layer's BF16 weights; both in the K-major canonical layout
// without swizzle (core matrices of 8 rows x 16 bytes: rows 16 bytes apart,
// the two K halves of an MMA 128 bytes apart, groups of 8 rows 256 bytes
// apart).  One thread issues the 18 MMAs into a 128 x 32 FP32 accumulator in
// tensor memory and commits them to an mbarrier; each warp then reads its 32
// rows (pixels) back with tcgen05.ld and writes the 32 channels, plus the
// bias and the ReLU.  The input-gradient convolution of the same layers is
// this kernel with the flipped, transposed weights.
constexpr int UM_M = 128;                          // pixels per CTA (MMA M)
constexpr int UM_N = 32;                           // output channels (MMA N)
constexpr int UM_KSTEPS = 9 * CNN_CMAX / 16;       // 18 MMAs of K = 16
constexpr int UM_A_STEP = UM_M * 16 * 2;           // bytes of A per MMA: 4096
constexpr int UM_B_STEP = UM_N * 16 * 2;           // bytes of B per MMA: 1024
constexpr size_t UM_SMEM = (size_t)UM_KSTEPS * (UM_A_STEP + UM_B_STEP) + 1024;   // + alignment slack
constexpr long long UM_WAIT_LIMIT = 1LL << 26;     // bounded wait on the MMAs' mbarrier

// tcgen05.mma instruction descriptor: D F32 (bits 4-5 = 1), A and B BF16
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28
constexpr uint32_t UM_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(UM_N >> 3) << 17) |
                              ((uint32_t)(UM_M >> 4) << 24);

// shared-memory matrix descriptor of a K-major operand without swizzle:
// start address, leading (K) and stride (8-row group) byte offsets, each in
// 16-byte units; version 1 at bit 46; layout type 0 (no swizzle) at bits 61-63
__device__ __forceinline__ uint64_t um_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t um_pack(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);   // a in the low half: the lower address
    return *reinterpret_cast<const uint32_t *>(&h);
}

__global__ void __launch_bounds__(UM_M) k_conv_umma(const float *__restrict__ in, const __nv_bfloat16 *__restrict__ w,
                                                    const float *__restrict__ b, float *__restrict__ out, int H, int W,
                                                    int relu, int *__restrict__ err)
{
    extern __shared__ unsigned char um_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_holder;
    unsigned char *As = reinterpret_cast<unsigned char *>(((uintptr_t)um_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *Bs = As + UM_KSTEPS * UM_A_STEP;
    const int t = threadIdx.x, warp = t >> 5;
    const long long plane = (long long)H * W;
    const long long p = (long long)blockIdx.x * UM_M + t;
    const bool live = p < plane;
    const int y = live ? (int)(p / W) : 0, x = live ? (int)(p % W) : 0;
    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(&mbar);

    if (warp == 0) {   // 32 columns of tensor memory: the 128 x 32 FP32 accumulator
        const uint32_t holder = (uint32_t)__cvta_generic_to_shared(&tmem_holder);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(holder) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A: the pixel's im2col row, 16 input channels of one tap per MMA
#pragma unroll 1
    for (int s = 0; s < UM_KSTEPS; s++) {
        const int tap = s >> 1, c0 = (s & 1) * 16;
        const int xx = x + tap % 3 - 1, yy = y + tap / 3 - 1;
        const bool ok = live && xx >= 0 && xx < W && yy >= 0 && yy < H;
        const size_t at = ok ? (size_t)c0 * (size_t)plane + (size_t)yy * W + xx : 0;
        uint32_t pk[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const float v0 = ok ? in[at + (size_t)(2 * e) * (size_t)plane] : 0.0f;
            const float v1 = ok ? in[at + (size_t)(2 * e + 1) * (size_t)plane] : 0.0f;
            pk[e] = um_pack(v0, v1);
        }
        unsigned char *row = As + s * UM_A_STEP + (t >> 3) * 256 + (t & 7) * 16;
        *reinterpret_cast<uint4 *>(row) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        *reinterpret_cast<uint4 *>(row + 128) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
    // B: w[co][ci][tap] as rows co of K = tap * 32 + ci, 16-byte chunks (step, co, half)
    for (int q = t; q < UM_KSTEPS * UM_N * 2; q += UM_M) {
        const int s = q >> 6, co = (q >> 1) & 31, half = q & 1;
        const int tap = s >> 1, c0 = (s & 1) * 16 + half * 8;
        uint16_t v[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const __nv_bfloat16 wv = w[(co * CNN_CMAX + c0 + e) * 9 + tap];
            v[e] = *reinterpret_cast<const uint16_t *>(&wv);
        }
        unsigned char *dst = Bs + s * UM_B_STEP + (co >> 3) * 256 + half * 128 + (co & 7) * 16;
        *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0] | ((uint32_t)v[1] << 16), v[2] | ((uint32_t)v[3] << 16),
                                                     v[4] | ((uint32_t)v[5] << 16), v[6] | ((uint32_t)v[7] << 16));
    }
    // the generic-proxy stores above become visible to the tensor cores' async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_holder;
    if (t == 0) {
        const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(As), b0 = (uint32_t)__cvta_generic_to_shared(Bs);
#pragma unroll 1
        for (int s = 0; s < UM_KSTEPS; s++) {
            const uint64_t ad = um_desc(a0 + s * UM_A_STEP, 128, 256), bd = um_desc(b0 + s * UM_B_STEP, 128, 256);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                         "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                         ::"r"(tmem), "l"(ad), "l"(bd), "r"(UM_IDESC), "r"(acc) : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                     : "memory");
    }
    // bounded wait for the MMAs (phase 0 of the mbarrier)
    int done = 0;
    for (long long it = 0; it < UM_WAIT_LIMIT && !done; it++) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(mbar_a), "r"(0u) : "memory");
        done = (int)ok;
    }
    done = __syncthreads_and(done);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                     "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                     "%30, %31}, [%32];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                       "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                       "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                       "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                     : "r"(taddr)
                     : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (live) {
#pragma unroll
            for (int co = 0; co < UM_N; co++) {
                float v = __uint_as_float(r[co]) + (b ? b[co] : 0.0f);
                if (relu && v < 0.0f) v = 0.0f;
                out[(size_t)co * (size_t)plane + (size_t)p] = v;
            }
        }
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}

// Weight gradient of a 32 -> 32 layer on the tensor cores: the GEMM
// D[m][co] = sum_p A[m][p] G[co][p] over the pixels, m = tap * 32 + ci
// (288 rows in three M = 128 tiles, the last one padded with zeros),
// A[m][p] = in[ci][p + tap] and G the layer's output gradient, both rounded to
// BF16.  Each CTA takes 128-pixel chunks of the plane (grid-stride), gathers
// them into shared memory in the K-major canonical layout (K = pixels),
// issues 3 x 8 MMAs per chunk into three 128 x 32 FP32 accumulators in tensor
// memory, and at the end writes its 288 x 32 partial sums; k_wgrad_reduce adds
// the CTAs' partials in a fixed order.
constexpr int UW_PIX = 128;                                   // pixels per chunk
constexpr int UW_TILES = 3;                                   // M tiles of 128 (288 rows)
constexpr int UW_A_TILE_STEP = UM_M * 16 * 2;                 // bytes of one tile for one MMA: 4096
constexpr int UW_A_BYTES = UW_TILES * (UW_PIX / 16) * UW_A_TILE_STEP;   // 98304
constexpr int UW_B_BYTES = (UW_PIX / 16) * UM_B_STEP;         // 8192
constexpr size_t UW_SMEM = (size_t)UW_A_BYTES + UW_B_BYTES + 1024;

__global__ void __launch_bounds__(UM_M) k_conv_wgrad_umma(const float *__restrict__ in, const float *__restrict__ g,
                                                          int H, int W, float *__restrict__ partial,
                                                          int *__restrict__ err)
{
    extern __shared__ unsigned char uw_raw[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_holder;
    unsigned char *As = reinterpret_cast<unsigned char *>(((uintptr_t)uw_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *Bs = As + UW_A_BYTES;
    const int t = threadIdx.x, warp = t >> 5;
    const long long plane = (long long)H * W;
    const long long nchunk = (plane + UW_PIX - 1) / UW_PIX;
    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(&mbar);
    if (warp == 0) {   // 3 x 32 columns: the three accumulators (allocated as 128)
        const uint32_t holder = (uint32_t)__cvta_generic_to_shared(&tmem_holder);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(holder) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows 288..383 (rows 32..127 of the last tile: row groups 4..15) stay zero
    for (int q = t; q < (UW_PIX / 16) * 12 * 2 * 8; q += UM_M) {   // steps x 12 row groups x 2 halves x 8 rows
        const int s = q / 192, rest = q % 192;
        unsigned char *dst = As + (2 * (UW_PIX / 16) + s) * UW_A_TILE_STEP + (4 + rest / 16) * 256 +
                             ((rest / 8) & 1) * 128 + (rest & 7) * 16;
        *reinterpret_cast<uint4 *>(dst) = make_uint4(0u, 0u, 0u, 0u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_holder;
    const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(As), b0 = (uint32_t)__cvta_generic_to_shared(Bs);
    int ok_all = 1;
    uint32_t phase = 0;
    bool first = true;
#pragma unroll 1
    for (long long c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const long long p0 = c * UW_PIX;
        // A: 288 rows (tap, ci) x 128 pixels, 16-byte chunks of 8 pixels
#pragma unroll 1
        for (int q = t; q < 288 * (UW_PIX / 8); q += UM_M) {
            const int m = q / (UW_PIX / 8), k8 = q % (UW_PIX / 8);
            const int tap = m >> 5, ci = m & 31, dx = tap % 3 - 1, dy = tap / 3 - 1;
            uint32_t pk[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                float v[2];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const long long pp = p0 + k8 * 8 + 2 * e + h;
                    v[h] = 0.0f;
                    if (pp < plane) {
                        const int y = (int)(pp / W) + dy, x = (int)(pp % W) + dx;
                        if (x >= 0 && x < W && y >= 0 && y < H) v[h] = in[(size_t)ci * plane + (size_t)y * W + x];
                    }
                }
                pk[e] = um_pack(v[0], v[1]);
            }
            const int tile = m >> 7, row = m & 127, s = k8 >> 1, half = k8 & 1;
            unsigned char *dst = As + (tile * (UW_PIX / 16) + s) * UW_A_TILE_STEP + (row >> 3) * 256 + half * 128 +
                                 (row & 7) * 16;
            *reinterpret_cast<uint4 *>(dst) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        // B: the output gradient, 32 rows (co) x 128 pixels
        for (int q = t; q < UM_N * (UW_PIX / 8); q += UM_M) {
            const int co = q / (UW_PIX / 8), k8 = q % (UW_PIX / 8);
            uint32_t pk[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const long long pp = p0 + k8 * 8 + 2 * e;
                const float v0 = pp < plane ? g[(size_t)co * plane + (size_t)pp] : 0.0f;
                const float v1 = pp + 1 < plane ? g[(size_t)co * plane + (size_t)pp + 1] : 0.0f;
                pk[e] = um_pack(v0, v1);
            }
            const int s = k8 >> 1, half = k8 & 1;
            unsigned char *dst = Bs + s * UM_B_STEP + (co >> 3) * 256 + half * 128 + (co & 7) * 16;
            *reinterpret_cast<uint4 *>(dst) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (t == 0) {
#pragma unroll 1
            for (int tile = 0; tile < UW_TILES; tile++)
#pragma unroll 1
                for (int s = 0; s < UW_PIX / 16; s++) {
                    const uint64_t ad = um_desc(a0 + (tile * (UW_PIX / 16) + s) * UW_A_TILE_STEP, 128, 256);
                    const uint64_t bd = um_desc(b0 + s * UM_B_STEP, 128, 256);
                    const uint32_t acc = (first && s == 0) ? 0u : 1u;
                    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                 ::"r"(tmem + (uint32_t)(tile * UM_N)), "l"(ad), "l"(bd), "r"(UM_IDESC), "r"(acc)
                                 : "memory");
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                         : "memory");
        }
        first = false;
        // the MMAs read the shared tiles: wait before the next chunk overwrites them
        int done = 0;
        for (long long it = 0; it < UM_WAIT_LIMIT && !done; it++) {
            uint32_t okw;
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(okw) : "r"(mbar_a), "r"(phase) : "memory");
            done = (int)okw;
        }
        phase ^= 1u;
        ok_all = __syncthreads_and(done);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok_all) break;
    }
    if (ok_all && !first) {
        float *out = partial + (size_t)blockIdx.x * 288 * UM_N;
#pragma unroll 1
        for (int tile = 0; tile < UW_TILES; tile++) {
            uint32_t r[32];
            const uint32_t taddr = tmem + (uint32_t)(tile * UM_N) + ((uint32_t)(warp * 32) << 16);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                         "%30, %31}, [%32];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                           "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                           "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                           "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                         : "r"(taddr)
                         : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int m = tile * UM_M + t;
            if (m < 288)
#pragma unroll
                for (int co = 0; co < UM_N; co++) out[(size_t)m * UM_N + co] = __uint_as_float(r[co]);
        }
    } else if (t == 0 && !ok_all) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
}

// dw[co][ci][tap] += sum over the CTAs (in order) of partial[cta][tap * 32 + ci][co]
__global__ void k_wgrad_reduce(const float *__restrict__ partial, int nparts, float *__restrict__ dw)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;   // q = m * 32 + co
    if (q >= 288 * UM_N) return;
    float s = 0.0f;
    for (int c = 0; c < nparts; c++) s += partial[(size_t)c * 288 * UM_N + q];
    const int m = q / UM_N, co = q % UM_N, tap = m >> 5, ci = m & 31;
    dw[(co * CNN_CMAX + ci) * 9 + tap] += s;
}

// the weights of the input-gradient convolution: wt[ci][co][8 - tap] = w[co][ci][tap]
__global__ void k_conv_transpose_weights(const __nv_bfloat16 *__restrict__ w, __nv_bfloat16 *__restrict__ wt,
                                         int cout, int cin)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= cout * cin * 9) return;
    const int co = q / (cin * 9), ci = (q / 9) % cin, t = q % 9;
    wt[(ci * cout + co) * 9 + (8 - t)] = w[q];
}

// dY *= (y > 0): the ReLU of a hidden layer, backwards
__global__ void k_relu_back(float *__restrict__ dy, const float *__restrict__ y, size_t n)
{
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n && !(y[q] > 0.0f)) dy[q] = 0.0f;
}

// weight and bias gradients of one layer: block (co, ci) sums
// in[ci][p + tap] * dY[co][p] over the pixels for the nine taps; block
// (co, cin) sums dY[co][p] for the bias
__global__ void __launch_bounds__(256) k_conv_wgrad(const float *__restrict__ in, int cin,
                                                    const float *__restrict__ dy, int H, int W,
                                                    float *__restrict__ dw, float *__restrict__ db)
{
    const int co = blockIdx.y, ci = blockIdx.x;
    const size_t plane = (size_t)H * W;
    const float *g = dy + co * plane;
    float acc[9];
#pragma unroll
    for (int t = 0; t < 9; t++) acc[t] = 0.0f;
    const bool bias = ci == cin;
    for (size_t p = threadIdx.x; p < plane; p += blockDim.x) {
        const float gv = g[p];
        if (gv == 0.0f) continue;
        if (bias) {
            acc[0] += gv;
            continue;
        }
        const int i = (int)(p % W), j = (int)(p / W);
        const float *x = in + ci * plane;
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const int a = i + t % 3 - 1, c = j + t / 3 - 1;
            if (a >= 0 && a < W && c >= 0 && c < H) acc[t] += x[(size_t)c * W + a] * gv;
        }
    }
    __shared__ float red[8][9];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < 9; t++) {
        float v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        float v = 0.0f;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) v += red[q][threadIdx.x];
        if (bias) {
            if (threadIdx.x == 0) db[co] += v;
        } else {
            dw[(co * cin + ci) * 9 + threadIdx.x] += v;
        }
    }
}

// mean-square loss and its gradient: dy = 2 (y - t) / n, loss partials per block
__global__ void k_mse(const float *__restrict__ y, const float *__restrict__ t, size_t n, float *__restrict__ dy,
                      double *__restrict__ loss)
{
    double s = 0.0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const float e = y[q] - t[q];
        dy[q] = 2.0f * e / (float)n;
        s += (double)e * (double)e;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (double)n);
}

// Adam (Kingma & Ba) on the FP32 master weights, then their BF16 copy
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       __nv_bfloat16 *__restrict__ wb, int n, float lr, float b1, float b2, float c1, float c2,
                       float eps)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float wq = w[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    w[q] = wq;
    wb[q] = __float2bfloat16(wq);
}

__global__ void k_to_bf16(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, int n)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) wb[q] = __float2bfloat16(w[q]);
}

// layer shapes of the fixed network and their offsets in the flat parameter
// array [w0, b0, w1, b1, ..., w5, b5] (w: [cout][cin][3][3])
struct Layer {
    int cin, cout;
    size_t w, b;   // offsets
};

constexpr int CNN_LAYERS = 6;
constexpr int CNN_IN = 3;

void layers(Layer (&L)[CNN_LAYERS])
{
    size_t off = 0;
    for (int l = 0; l < CNN_LAYERS; l++) {
        L[l].cin = l == 0 ? CNN_IN : CNN_CMAX;
        L[l].cout = l == CNN_LAYERS - 1 ? 1 : CNN_CMAX;
        L[l].w = off;
        off += (size_t)L[l].cout * L[l].cin * 9;
        L[l].b = off;
        off += (size_t)L[l].cout;
    }
}

size_t param_count()
{
    Layer L[CNN_LAYERS];
    layers(L);
    return L[CNN_LAYERS - 1].b + 1;
}

// activation planes kept in the work buffer: the five hidden layers' outputs
// (32 planes each) and the output plane, then two gradient buffers of 32
// planes, then the transposed weights of one layer
__device__ int g_cnn_err;   // set when a tensor-core convolution gave up waiting for its MMAs

constexpr int UW_MAX_CTAS = 296;   // tensor-core weight-gradient CTAs (two per SM of a B200)

size_t work_floats(int H, int W)
{
    const size_t plane = (size_t)H * W;
    return (5 * CNN_CMAX + 1 + 2 * CNN_CMAX) * plane + CNN_CMAX * CNN_CMAX * 9 + (size_t)UW_MAX_CTAS * 288 * UM_N;
}

// weight and bias gradient of a 32 -> 32 layer: the weights on the tensor
// cores, the bias by per-block sums
int wgrad32(const float *in, const float *g, float *dw, float *db, int H, int W, float *partial, cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv_wgrad_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UW_SMEM) !=
            cudaSuccess)
            return -1;
        attr = true;
    }
    int *err = nullptr;
    if (cudaGetSymbolAddress((void **)&err, g_cnn_err) != cudaSuccess) return -1;
    const long long n = (long long)H * W, nchunk = (n + UW_PIX - 1) / UW_PIX;
    const int nb = (int)(nchunk < UW_MAX_CTAS ? nchunk : UW_MAX_CTAS);   // every CTA gets a chunk
    k_conv_wgrad_umma<<<(unsigned)nb, UM_M, UW_SMEM, st>>>(in, g, H, W, partial, err);
    k_wgrad_reduce<<<(288 * UM_N + 255) / 256, 256, 0, st>>>(partial, nb, dw);
    k_conv_wgrad<<<dim3(1u, (unsigned)CNN_CMAX), 256, 0, st>>>(in, 0, g, H, W, dw, db);   // bias only
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

size_t conv_smem(int cin, int cout) { return sizeof(float) * ((size_t)cin * CNN_HALO * CNN_HALO + (size_t)cout * cin * 9); }

int conv(const float *in, int cin, const __nv_bfloat16 *w, const float *b, float *out, int cout, int H, int W, int relu,
         cudaStream_t st)
{
    if (cin == CNN_CMAX && cout == CNN_CMAX) {   // the hidden layers: tensor cores
        static bool um_attr = false;
        if (!um_attr) {
            if (cudaFuncSetAttribute(k_conv_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UM_SMEM) !=
                cudaSuccess)
                return -1;
            um_attr = true;
        }
        int *err = nullptr;
        if (cudaGetSymbolAddress((void **)&err, g_cnn_err) != cudaSuccess) return -1;
        const long long n = (long long)H * W;
        k_conv_umma<<<(unsigned)((n + UM_M - 1) / UM_M), UM_M, UM_SMEM, st>>>(in, w, b, out, H, W, relu, err);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    }
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_conv3x3<CNN_CMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)conv_smem(CNN_CMAX, CNN_CMAX)) != cudaSuccess ||
            cudaFuncSetAttribute(k_conv3x3<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)conv_smem(CNN_CMAX, 1)) != cudaSuccess)
            return -1;
        attr = true;
    }
    const dim3 grd((unsigned)((W + CNN_TILE - 1) / CNN_TILE), (unsigned)((H + CNN_TILE - 1) / CNN_TILE));
    const size_t sm = conv_smem(cin, cout);
    if (cout == CNN_CMAX) k_conv3x3<CNN_CMAX><<<grd, CNN_TILE * CNN_TILE, sm, st>>>(in, cin, w, b, out, H, W, relu);
    else if (cout == 1) k_conv3x3<1><<<grd, CNN_TILE * CNN_TILE, sm, st>>>(in, cin, w, b, out, H, W, relu);
    else return -1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

// sums of squares over the physical cells (W x H) of two planes, per block
__global__ void k_cnn_sumsq(Dom d, const double *__restrict__ a, const double *__restrict__ b,
                            double *__restrict__ partials)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    double sa = 0.0, sb = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < W * H; q += gridDim.x * blockDim.x) {
        const int i = q % W, j = q / W;
        const double x = AT_(a, i, j), y = AT_(b, i, j);
        sa += x * x;
        sb += y * y;
    }
    __shared__ double sh[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_down_sync(0xffffffffu, sa, o);
        sb += __shfl_down_sync(0xffffffffu, sb, o);
    }
    if (lane == 0) { sh[0][warp] = sa; sh[1][warp] = sb; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sh[threadIdx.x][q];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

// the residual of the previous correction under this substep's right-hand
// side, r0 = rhs - A phi_prev (A: the variable-density operator of the
// pressure solve with its ghost update), on the physical cells
__global__ void k_cnn_residual(Dom d, BcMap mp, const double *__restrict__ rho, const double *__restrict__ rhs,
                               const double *__restrict__ phi_prev, double *__restrict__ r0)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= W * H) return;
    const int i = q % W, j = q / W;
    const double a = pressure_op(d, rho, i, j, [&](int x, int y) { return remap(mp, phi_prev, P, d.NX, d.NY, x, y); });
    // the right-hand side with the operator's axisymmetric row weight, as the solve forms its residual
    AT_(r0, i, j) = (d.axisym ? AT_(rhs, i, j) * d.m.r_c[i] : AT_(rhs, i, j)) - a;
}

// network inputs x = [rho, r0 / rms(r0), phi_prev / rms(phi_prev)] and, if
// phi is given, the target t = (phi - phi_prev) / rms(phi_prev)
__global__ void k_cnn_assemble(Dom d, const double *__restrict__ rho, const double *__restrict__ rhs,
                               const double *__restrict__ phi_prev, const double *__restrict__ phi,
                               const DevScalars *__restrict__ sc, float *__restrict__ x, float *__restrict__ t)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= W * H) return;
    const int i = q % W, j = q / W;
    const double n = (double)W * H;
    const double rr = sqrt(sc->cnn_ms[0] / n) + 1e-300, rp = sqrt(sc->cnn_ms[1] / n) + 1e-300;
    const size_t plane = (size_t)W * H;
    x[q] = (float)AT_(rho, i, j);
    x[plane + q] = (float)(AT_(rhs, i, j) / rr);
    x[2 * plane + q] = (float)(AT_(phi_prev, i, j) / rp);
    if (phi) t[q] = (float)((AT_(phi, i, j) - AT_(phi_prev, i, j)) / rp);
}

// the network's change as a plane of the solve's layout: e = y (ghosts zero)
__global__ void k_cnn_expand(Dom d, const float *__restrict__ y, double *__restrict__ e)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= W * H) return;
    AT_(e, q % W, q / W) = (double)y[q];
}

// the two inner products of the step along e that minimises the residual in
// the solve's stopping norm (r . M r, M the Jacobi preconditioner): per block
// sum (A e) M r0 and sum (A e) M (A e) over the physical cells
__global__ void k_cnn_galerkin(Dom d, BcMap mp, const double *__restrict__ rho, const double *__restrict__ e,
                               const double *__restrict__ r0, const double *__restrict__ M, double *__restrict__ partials)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    double s0 = 0.0, s1 = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < W * H; q += gridDim.x * blockDim.x) {
        const int i = q % W, j = q / W;
        const double ae = pressure_op(d, rho, i, j, [&](int x, int y) { return remap(mp, e, P, d.NX, d.NY, x, y); });
        const double m = AT_(M, i, j);
        s0 += ae * m * AT_(r0, i, j);
        s1 += ae * m * ae;
    }
    __shared__ double sh[2][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
    }
    if (lane == 0) { sh[0][warp] = s0; sh[1][warp] = s1; }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sh[threadIdx.x][q];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

// the warm start phi = phi_prev + alpha e with alpha = (A e . M r0) /
// (A e . M A e): of the corrections along e it leaves the smallest residual
// in the solve's stopping norm, so the solve never starts further from its
// stopping test than from phi_prev
__global__ void k_cnn_apply(Dom d, const double *__restrict__ e, const double *__restrict__ phi_prev,
                            const DevScalars *__restrict__ sc, double *__restrict__ phi)
{
    const int W = d.NX - 1, H = d.NY - 1, P = d.P;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= W * H) return;
    const int i = q % W, j = q / W;
    const double den = sc->cnn_ms[1];
    const double alpha = (den != 0.0) ? sc->cnn_ms[0] / den : 0.0;
    AT_(phi, i, j) = AT_(phi_prev, i, j) + alpha * AT_(e, i, j);
}

}  // namespace pvof

using namespace pvof;

extern "C" {

size_t pvof_cnn_param_count(void) { return param_count(); }

size_t pvof_cnn_work_floats(int H, int W) { return (H > 0 && W > 0) ? work_floats(H, W) : 0; }

int pvof_cnn_forward(const float *params, const uint16_t *params_bf16, const float *x, float *y, int H, int W,
                     float *work, void *stream)
{
    if (!params || !params_bf16 || !x || !work || H <= 0 || W <= 0) return PVOF_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    Layer L[CNN_LAYERS];
    layers(L);
    const size_t plane = (size_t)H * W;
    const __nv_bfloat16 *wb = reinterpret_cast<const __nv_bfloat16 *>(params_bf16);
    const float *in = x;
    for (int l = 0; l < CNN_LAYERS; l++) {
        float *out = work + (size_t)l * CNN_CMAX * plane;   // layer l's output (the last: one plane)
        if (conv(in, L[l].cin, wb + L[l].w, params + L[l].b, out, L[l].cout, H, W, l < CNN_LAYERS - 1, st))
            return PVOF_ECUDA;
        in = out;
    }
    if (y && cudaMemcpyAsync(y, in, plane * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return PVOF_ECUDA;
    return PVOF_OK;
}

int pvof_cnn_backward(const float *params, const uint16_t *params_bf16, const float *x, const float *dy, float *grad,
                      int H, int W, float *work, void *stream)
{
    if (!params || !params_bf16 || !x || !dy || !grad || !work || H <= 0 || W <= 0) return PVOF_EINVAL;
    (void)params;
    cudaStream_t st = (cudaStream_t)stream;
    Layer L[CNN_LAYERS];
    layers(L);
    const size_t plane = (size_t)H * W;
    const __nv_bfloat16 *wb = reinterpret_cast<const __nv_bfloat16 *>(params_bf16);
    float *gbuf[2] = {work + (5 * CNN_CMAX + 1) * plane, work + (6 * CNN_CMAX + 1) * plane};
    __nv_bfloat16 *wt = reinterpret_cast<__nv_bfloat16 *>(work + (7 * CNN_CMAX + 1) * plane);
    float *partial = work + (7 * CNN_CMAX + 1) * plane + CNN_CMAX * CNN_CMAX * 9;
    // gradient at the output of the last layer
    if (cudaMemcpyAsync(gbuf[0], dy, plane * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return PVOF_ECUDA;
    int cur = 0;
    for (int l = CNN_LAYERS - 1; l >= 0; l--) {
        const float *lin = l == 0 ? x : work + (size_t)(l - 1) * CNN_CMAX * plane;
        float *g = gbuf[cur];
        if (l < CNN_LAYERS - 1) {   // through this layer's ReLU
            const size_t n = (size_t)L[l].cout * plane;
            k_relu_back<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, work + (size_t)l * CNN_CMAX * plane, n);
        }
        if (L[l].cin == CNN_CMAX && L[l].cout == CNN_CMAX) {   // a tensor-core layer
            if (wgrad32(lin, g, grad + L[l].w, grad + L[l].b, H, W, partial, st)) return PVOF_ECUDA;
        } else {
            k_conv_wgrad<<<dim3((unsigned)L[l].cin + 1, (unsigned)L[l].cout), 256, 0, st>>>(
                lin, L[l].cin, g, H, W, grad + L[l].w, grad + L[l].b);
        }
        if (l > 0) {   // gradient at this layer's input: the flipped, transposed convolution
            const int n = L[l].cout * L[l].cin * 9;
            k_conv_transpose_weights<<<(n + 255) / 256, 256, 0, st>>>(wb + L[l].w, wt, L[l].cout, L[l].cin);
            if (conv(g, L[l].cout, wt, nullptr, gbuf[1 - cur], L[l].cin, H, W, 0, st)) return PVOF_ECUDA;
            cur = 1 - cur;
        }
    }
    return cudaGetLastError() == cudaSuccess ? PVOF_OK : PVOF_ECUDA;
}

int pvof_cnn_mse(const float *y, const float *t, float *dy, size_t n, double *loss, void *stream)
{
    if (!y || !t || !dy || !loss || n == 0) return PVOF_EINVAL;
    k_mse<<<296, 256, 0, (cudaStream_t)stream>>>(y, t, n, dy, loss);
    return cudaGetLastError() == cudaSuccess ? PVOF_OK : PVOF_ECUDA;
}

int pvof_cnn_adam(float *params, const float *grad, float *m, float *v, uint16_t *params_bf16, int step, float lr,
                  void *stream)
{
    if (!params || !grad || !m || !v || !params_bf16 || step < 1) return PVOF_EINVAL;
    const int n = (int)param_count();
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v,
                                                             reinterpret_cast<__nv_bfloat16 *>(params_bf16), n, lr, b1,
                                                             b2, c1, c2, 1e-8f);
    return cudaGetLastError() == cudaSuccess ? PVOF_OK : PVOF_ECUDA;
}

int pvof_cnn_conv32(const float *x, const uint16_t *w_bf16, const float *b, float *y, int H, int W, int relu,
                    void *stream)
{
    if (!x || !w_bf16 || !y || H <= 0 || W <= 0) return PVOF_EINVAL;
    return conv(x, CNN_CMAX, reinterpret_cast<const __nv_bfloat16 *>(w_bf16), b, y, CNN_CMAX, H, W, relu,
                (cudaStream_t)stream)
               ? PVOF_ECUDA
               : PVOF_OK;
}

int pvof_cnn_status(void *stream)
{
    int *err = nullptr, h = 0;
    if (cudaGetSymbolAddress((void **)&err, g_cnn_err) != cudaSuccess) return PVOF_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PVOF_ECUDA;
    if (h && cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return PVOF_ECUDA;
    return h ? PVOF_ECUDA : PVOF_OK;
}

int pvof_cnn_to_bf16(const float *params, uint16_t *params_bf16, void *stream)
{
    if (!params || !params_bf16) return PVOF_EINVAL;
    const int n = (int)param_count();
    k_to_bf16<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, reinterpret_cast<__nv_bfloat16 *>(params_bf16),
                                                                 n);
    return cudaGetLastError() == cudaSuccess ? PVOF_OK : PVOF_ECUDA;
}

}  // extern "C"
