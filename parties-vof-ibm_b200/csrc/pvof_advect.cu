// VOF_DIFFUSE_advect_WENO5 (Eulerian/VOF_DIFFUSE.c:931-996) as one kernel:
// the WENO5 face fluxes (:453-498, :958-973), their ghost update
// (Velocity_update_boundaries on the flux arrays) and the flux divergence
// (TwodOps_scalar_flux_divergence, TwodOps.c:201-229) per tile, with the
// tiles of C_L, u and v brought into shared memory by the tensor memory
// accelerator (cp.async.bulk.tensor, no multicast) behind an mbarrier.
//
// A tile is 32 x 8 cells.  Its face fluxes (33 x 8 x faces, 32 x 9 y faces)
// are computed once into shared memory and the divergence of every cell read
// from there.  Each face flux is the same expression on the same operands as
// the separate flux kernel, so the fluxes, and the divergence, are bit for
// bit those of the three-launch form.  A face on the ghost frame whose ghost
// rule is not the identity takes the rule's value (mul_x mul_y times the flux
// at the source face, computed from global memory), as the ghost update of
// the flux arrays gives it.
//
// TMA rules kept: the boxes start at an even column (the first column of a
// tile's box is the plane column OX + i0 - 4 = i0, with i0 a multiple of 32),
// so x times 8 bytes is a multiple of 16; box widths are 40 doubles (320
// bytes); the plane's row stride is a multiple of 32 doubles; columns or rows
// past the plane read the fill value (zero) and feed no computed face.  The
// wait on the mbarrier is bounded: on timeout the kernel records error code 4
// in DevScalars and its tile writes nothing.
#include <cuda.h>

#include "pvof_device.cuh"
#include "pvof_kernels.cuh"

namespace pvof {

namespace {

constexpr int ADV_TX = 32, ADV_TY = 8;
constexpr int ADV_W = ADV_TX + 8;                  // box width: 4 columns left of the tile, 4 right
constexpr int ADV_CROWS = ADV_TY + 6, ADV_UROWS = ADV_TY, ADV_VROWS = ADV_TY + 1;
constexpr long long ADV_WAIT_LIMIT = 1LL << 26;
constexpr unsigned ADV_BYTES = (ADV_CROWS + ADV_UROWS + ADV_VROWS) * ADV_W * sizeof(double);

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(d), "l"(map), "r"(x), "r"(y), "r"(bar) : "memory");
}

// WENO5 (or upwind) state of a face from the five cells c(-3) .. c(+1) about
// it, upwinded by the sign of the face velocity; the flux vel * state
template <bool FP32, class Cget>
__device__ __forceinline__ double face_flux(double vel, int weno5, Cget c)
{
    if (FP32) {
        const float vf = (float)vel;
        float st;
        if (weno5) st = (vf >= 0.0f) ? weno5_left_f((float)c(-3), (float)c(-2), (float)c(-1), (float)c(0), (float)c(1))
                                     : weno5_left_f((float)c(2), (float)c(1), (float)c(0), (float)c(-1), (float)c(-2));
        else st = (vf >= 0.0f) ? (float)c(-1) : (float)c(0);
        return (double)(vf * st);
    }
    double st;
    if (weno5) st = (vel >= 0.0) ? weno5_left(c(-3), c(-2), c(-1), c(0), c(1)) : weno5_left(c(2), c(1), c(0), c(-1), c(-2));
    else st = (vel >= 0.0) ? c(-1) : c(0);
    return vel * st;
}

// the x-face flux at (i, j) from global memory (ghost-frame faces)
template <bool FP32>
__device__ double xflux_global(const Dom &d, const double *C, const double *u, int weno5, int i, int j)
{
    const int P = d.P;
    return face_flux<FP32>(AT_(u, i, j), weno5, [&](int o) { return AT_(C, i + o, j); });
}

template <bool FP32>
__device__ double yflux_global(const Dom &d, const double *C, const double *v, int weno5, int i, int j)
{
    const int P = d.P;
    return face_flux<FP32>(AT_(v, i, j), weno5, [&](int o) { return AT_(C, i, j + o); });
}

template <bool FP32>
__global__ void __launch_bounds__(ADV_TX * ADV_TY)
    k_advect_tma(Dom d, BcMap mu, BcMap mv, const __grid_constant__ CUtensorMap tmC,
                 const __grid_constant__ CUtensorMap tmU, const __grid_constant__ CUtensorMap tmV,
                 const double *__restrict__ C, const double *__restrict__ u, const double *__restrict__ v, int weno5,
                 double *__restrict__ out, DevScalars *scal)
{
    __shared__ __align__(128) double sC[ADV_CROWS * ADV_W];
    __shared__ __align__(128) double sU[ADV_UROWS * ADV_W];
    __shared__ __align__(128) double sV[ADV_VROWS * ADV_W];
    __shared__ double fxs[ADV_TY][ADV_TX + 1], fys[ADV_TY + 1][ADV_TX];
    __shared__ __align__(8) unsigned long long bar;
    const int tid = threadIdx.y * ADV_TX + threadIdx.x;
    const int i0 = blockIdx.x * ADV_TX, j0 = blockIdx.y * ADV_TY;
    const int NX = d.NX, NY = d.NY, P = d.P;
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(ADV_BYTES) : "memory");
        tma_load_2d(sC, &tmC, OX + i0 - 4, OY + j0 - 3, b);
        tma_load_2d(sU, &tmU, OX + i0 - 4, OY + j0, b);
        tma_load_2d(sV, &tmV, OX + i0 - 4, OY + j0, b);
    }
    int done = 0;
    for (long long it = 0; it < ADV_WAIT_LIMIT && !done; it++) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(b), "r"(0u) : "memory");
        done = (int)ok;
    }
    done = __syncthreads_and(done);
    if (!done) {
        if (tid == 0) atomicCAS(&scal->error, 0, 4);   // 4: an advection tile load gave up
        return;
    }
    // face fluxes of the tile
    for (int e = tid; e < ADV_TY * (ADV_TX + 1); e += ADV_TX * ADV_TY) {
        const int r = e / (ADV_TX + 1), cx = e - r * (ADV_TX + 1), i = i0 + cx, j = j0 + r;
        if (j >= NY || i > NX) continue;
        const int si = mu.x.src[i + NG], sj = mu.y.src[j + NG];
        const double mx = mu.x.mul[i + NG], my = mu.y.mul[j + NG];
        double f;
        if (si == i && sj == j && mx == 1.0 && my == 1.0) {
            // (the face past the last cell with an identity rule is never
            // written by the three-launch form: its scratch keeps zero)
            if (i == NX) { fxs[r][cx] = 0.0; continue; }
            const double *row = sC + (r + 3) * ADV_W + cx + 4;
            f = face_flux<FP32>(sU[r * ADV_W + cx + 4], weno5, [&](int o) { return row[o]; });
        } else {
            f = (mx != 0.0 && my != 0.0) ? mx * my * xflux_global<FP32>(d, C, u, weno5, si, sj) : 0.0;
        }
        fxs[r][cx] = f;
    }
    for (int e = tid; e < (ADV_TY + 1) * ADV_TX; e += ADV_TX * ADV_TY) {
        const int r = e / ADV_TX, cx = e - r * ADV_TX, i = i0 + cx, j = j0 + r;
        if (i >= NX || j > NY) continue;
        const int si = mv.x.src[i + NG], sj = mv.y.src[j + NG];
        const double mx = mv.x.mul[i + NG], my = mv.y.mul[j + NG];
        double f;
        if (si == i && sj == j && mx == 1.0 && my == 1.0) {
            if (j == NY) { fys[r][cx] = 0.0; continue; }
            const double *col = sC + (r + 3) * ADV_W + cx + 4;
            f = face_flux<FP32>(sV[r * ADV_W + cx + 4], weno5, [&](int o) { return col[o * ADV_W]; });
        } else {
            f = (mx != 0.0 && my != 0.0) ? mx * my * yflux_global<FP32>(d, C, v, weno5, si, sj) : 0.0;
        }
        fys[r][cx] = f;
    }
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y, i = i0 + tx, j = j0 + ty;
    if (i >= NX || j >= NY) return;
    const double fx0 = fxs[ty][tx], fx1 = fxs[ty][tx + 1];
    const double div_x = (fx1 - fx0) / d.m.dx_c[i];
    const double div_y = (fys[ty + 1][tx] - fys[ty][tx]) / d.m.dy_c[j];
    double div;
    if (d.planar) div = div_x + div_y;
    else div = (d.m.r_u[i + 1] * fx1 - d.m.r_u[i] * fx0) * d.m.inv_r_c[i] / d.m.dx_c[i] + div_y;
    AT_(out, i, j) = -div;
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiled)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// a tensor map over a whole ghosted plane (P x (NY + 2 NG) doubles) with a
// box of ADV_W x rows
bool plane_map(CUtensorMap *m, const double *base, int P, int rows_total, int box_rows)
{
    EncodeTiled enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)rows_total};
    const cuuint64_t strides[1] = {(cuuint64_t)P * sizeof(double)};
    const cuuint32_t box[2] = {(cuuint32_t)ADV_W, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

struct AdvectMaps {
    CUtensorMap c, u, v;
};

// the tensor maps of a context's C_L, u and v planes (their storage never
// moves); null when the driver offers no tensor-map encoder
AdvectMaps *advect_maps_create(const double *C_base, const double *u_base, const double *v_base, int P, int NY)
{
    AdvectMaps *a = new AdvectMaps();
    const int rows = NY + 2 * NG;
    if (!plane_map(&a->c, C_base, P, rows, ADV_CROWS) || !plane_map(&a->u, u_base, P, rows, ADV_UROWS) ||
        !plane_map(&a->v, v_base, P, rows, ADV_VROWS)) {
        delete a;
        return nullptr;
    }
    return a;
}

void advect_maps_destroy(AdvectMaps *a) { delete a; }

cudaError_t advect_tma_launch(const AdvectMaps *a, const Dom &d, const BcMap &mu, const BcMap &mv, const double *C,
                              const double *u, const double *v, int weno5, bool fp32, double *out, DevScalars *scal,
                              cudaStream_t st)
{
    const dim3 blk(ADV_TX, ADV_TY), grd((unsigned)((d.NX + ADV_TX - 1) / ADV_TX), (unsigned)((d.NY + ADV_TY - 1) / ADV_TY));
    if (fp32) k_advect_tma<true><<<grd, blk, 0, st>>>(d, mu, mv, a->c, a->u, a->v, C, u, v, weno5, out, scal);
    else k_advect_tma<false><<<grd, blk, 0, st>>>(d, mu, mv, a->c, a->u, a->v, C, u, v, weno5, out, scal);
    return cudaGetLastError();
}

}  // namespace pvof
