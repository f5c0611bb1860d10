// pvof_Pressure_solve_cg_noalloc: the variable-density pressure solve
// (Jacobi preconditioner + Jacobi PCG + ghost update of the correction) for
// callers that cannot allocate device memory -- code that runs where
// cudaMalloc is not available to it, such as a host solver that hands the
// library buffers from its own fixed device pool or runs inside a region
// where allocation calls are not allowed.  The caller owns the inputs and the
// output; every temporary this solve needs lives in one fixed-size device
// array declared in this file, so the entry point itself allocates nothing.
//
// Limits and sharing:
//   * the scratch holds planes of at most NOALLOC_PLANE_MAX doubles, i.e.
//     (NXM+7)*(NYM+7) <= NOALLOC_PLANE_MAX, and NXM, NYM <= NOALLOC_AXIS_MAX;
//     larger grids are rejected with PVOF_EINVAL;
//   * the array is statically allocated on every GPU that loads the library
//     and stays allocated until the process exits (about 3.7 MB);
//   * every call on a device uses the same array and leaves its contents
//     behind; calls that overlap on the GPU (different streams or threads,
//     same device) race on it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
#include <cmath>
#include <cstring>
#include <mutex>

#include "pvof_kernels.cuh"

namespace pvof {

constexpr size_t NOALLOC_PLANE_MAX = 72000;
constexpr int NOALLOC_AXIS_MAX = 1024;
constexpr int NOALLOC_THREADS = 512;
constexpr int NOALLOC_MAX_BLOCKS = 8 * 160;
constexpr size_t NOALLOC_AXIS_LEN = NOALLOC_AXIS_MAX + 1 + 2 * NG;  // entries of a per-axis table

// layout of the scratch array, in doubles
constexpr size_t NA_PLANES = 6;  // M, res, dir, dir2, z, Ad
constexpr size_t NA_OFF_PART = NA_PLANES * NOALLOC_PLANE_MAX;
constexpr size_t NA_OFF_SCAL = NA_OFF_PART + 4 * (size_t)NOALLOC_MAX_BLOCKS;
constexpr size_t NA_SCAL_LEN = (sizeof(DevScalars) + sizeof(double) - 1) / sizeof(double);
constexpr size_t NA_OFF_METRIC = NA_OFF_SCAL + NA_SCAL_LEN;
constexpr size_t NA_NMETRIC = 6;  // idx_c, idy_c, r_u, r_c, inv_r_c, zeros
constexpr size_t NA_OFF_MAPMUL = NA_OFF_METRIC + NA_NMETRIC * NOALLOC_AXIS_LEN;
constexpr size_t NA_NMAP = 4;  // pressure x/y, scalar exchange x/y
constexpr size_t NA_OFF_MAPSRC = NA_OFF_MAPMUL + NA_NMAP * NOALLOC_AXIS_LEN;  // ints packed two per double
constexpr size_t NA_TOTAL = NA_OFF_MAPSRC + (NA_NMAP * NOALLOC_AXIS_LEN + 1) / 2;

static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL];

namespace {

struct DeviceScratch {
    double *base = nullptr;
    int coop_blocks = 0;
};

std::mutex g_mu;
DeviceScratch g_dev[64];

int na_err(int code, const char *msg);

// per-device set-up: device address of the scratch array and the
// co-resident block count of the grid-wide pressure solver
int scratch_for_device(int dev, DeviceScratch &out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= 64) return na_err(PVOF_EINVAL, "device index out of range");
    DeviceScratch &s = g_dev[dev];
    if (!s.base) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return na_err(PVOF_ECUDA, "cudaGetSymbolAddress of the scratch array failed");
        int nsm = 0, occ = 0;
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cg_pressure, NOALLOC_THREADS, 0) != cudaSuccess || occ < 1)
            return na_err(PVOF_ECUDA, "occupancy query failed");
        int nb = occ * nsm;
        s.coop_blocks = nb < NOALLOC_MAX_BLOCKS ? nb : NOALLOC_MAX_BLOCKS;
        s.base = (double *)p;
    }
    out = s;
    return PVOF_OK;
}

thread_local const char *g_na_msg = "";
int na_err(int code, const char *msg)
{
    g_na_msg = msg;
    return code;
}

// host copies of the tables the pressure kernels read (built as pvof_create
// builds them: PARTIES/src/Grid.c:797-918, psolve_cg.c:358-529,
// Communication.c:146-291)
struct HostTables {
    double metric[NA_NMETRIC][NOALLOC_AXIS_LEN];
    double mul[NA_NMAP][NOALLOC_AXIS_LEN];
    int src[NA_NMAP][NOALLOC_AXIS_LEN];
};
thread_local HostTables g_tab;

void build_tables(const pvof_grid_desc &g, int NX, int NY)
{
    std::memset(&g_tab, 0, sizeof(g_tab));
    const double dx = (g.xmax - g.xmin) / (double)(NX - 1), dy = (g.ymax - g.ymin) / (double)(NY - 1);
    for (int i = -NG; i < NX + NG - 1; i++) {
        double xc0 = g.xmin + (0.5 + i) * dx, xc1 = g.xmin + (0.5 + (i + 1)) * dx;
        g_tab.metric[0][i + NG] = 1.0 / (xc1 - xc0);
    }
    for (int j = -NG; j < NY + NG - 1; j++) {
        double yc0 = g.ymin + (0.5 + j) * dy, yc1 = g.ymin + (0.5 + (j + 1)) * dy;
        g_tab.metric[1][j + NG] = 1.0 / (yc1 - yc0);
    }
    if (g.geometry == PVOF_GEOM_AXISYM) {
        for (int i = -NG; i < NX + NG; i++) {
            double ru = std::fabs(g.xmin + i * dx), rc = std::fabs(g.xmin + (0.5 + i) * dx);
            g_tab.metric[2][i + NG] = ru;
            g_tab.metric[3][i + NG] = rc;
            g_tab.metric[4][i + NG] = (rc > 1.0e-14) ? 1.0 / rc : 0.0;
        }
    }
    // maps: 0 pressure x, 1 pressure y, 2 exchange x, 3 exchange y
    const int N[4] = {NX, NY, NX, NY};
    const bool per[4] = {g.periodic[0] != 0, g.periodic[1] != 0, g.periodic[0] != 0, g.periodic[1] != 0};
    for (int m = 0; m < 4; m++) {
        for (int i = -NG; i < N[m] + NG; i++) {
            g_tab.src[m][i + NG] = i;
            g_tab.mul[m][i + NG] = 1.0;
        }
        if (per[m]) {
            for (int i = -NG; i <= -1; i++) g_tab.src[m][i + NG] = i + (N[m] - 1);
            for (int i = N[m] - 1; i <= N[m] + 1; i++) g_tab.src[m][i + NG] = i - (N[m] - 1);
        } else if (m < 2) {
            g_tab.src[m][-1 + NG] = 0;
            g_tab.src[m][N[m] - 1 + NG] = N[m] - 2;
        }
    }
}

}  // namespace
}  // namespace pvof

using namespace pvof;

extern "C" const char *pvof_noalloc_last_error(void) { return g_na_msg; }

// See the file comment and include/pvof.h.
extern "C" int pvof_Pressure_solve_cg_noalloc(const pvof_grid_desc *grid, const pvof_params *params,
                                              const double *rho, const double *rhs, double *phi, void *stream,
                                              int *iterations, double *residual)
{
    if (!grid || !params || !rho || !rhs || !phi) return na_err(PVOF_EINVAL, "null argument");
    if (grid->ghost_nodes != NG || grid->NZM != 1 ||
        (grid->geometry != PVOF_GEOM_PLANAR && grid->geometry != PVOF_GEOM_AXISYM))
        return na_err(PVOF_EINVAL, "needs a 2D grid with 3 ghost layers");
    if (grid->geometry == PVOF_GEOM_AXISYM && grid->periodic[0])
        return na_err(PVOF_EINVAL, "an axisymmetric grid has the symmetry axis on its left: x cannot be periodic");
    if (grid->NXM < 8 || grid->NYM < 8 || grid->NXM > NOALLOC_AXIS_MAX || grid->NYM > NOALLOC_AXIS_MAX ||
        (size_t)(grid->NXM + 7) * (size_t)(grid->NYM + 7) > NOALLOC_PLANE_MAX)
        return na_err(PVOF_EINVAL, "grid exceeds the fixed scratch: (NXM+7)*(NYM+7) must be <= 72000 "
                                   "and NXM, NYM <= 1024");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return na_err(PVOF_ENODEV, "no CUDA device");
    DeviceScratch sc;
    int rc = scratch_for_device(dev, sc);
    if (rc != PVOF_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int NX = grid->NXM + 1, NY = grid->NYM + 1;

    // domain over the caller's planes: row stride NX+6, element (0,0) at (3,3)
    Dom d;
    std::memset(&d, 0, sizeof(d));
    d.NX = NX;
    d.NY = NY;
    d.P = NX + 2 * NG;
    d.planar = grid->geometry == PVOF_GEOM_PLANAR;
    d.axisym = grid->geometry == PVOF_GEOM_AXISYM;
    d.perx = grid->periodic[0] != 0;
    d.pery = grid->periodic[1] != 0;
    d.nk = 2;
    d.slab = grid->slab_thickness;
    d.wz = d.planar ? d.slab : 1.0;
    double *base = sc.base;
    double *metric = base + NA_OFF_METRIC;
    const double *zeros = metric + 5 * NOALLOC_AXIS_LEN + NG;
    d.m.idx_c = metric + 0 * NOALLOC_AXIS_LEN + NG;
    d.m.idy_c = metric + 1 * NOALLOC_AXIS_LEN + NG;
    d.m.r_u = metric + 2 * NOALLOC_AXIS_LEN + NG;
    d.m.r_c = metric + 3 * NOALLOC_AXIS_LEN + NG;
    d.m.inv_r_c = metric + 4 * NOALLOC_AXIS_LEN + NG;
    d.m.idx_u = d.m.dx_c = d.m.dx_u = d.m.idy_v = d.m.dy_c = d.m.dy_v = zeros;
    d.m.inv_r_u = d.m.ring_wt_c = d.m.wx = d.m.wy = zeros;
    double *mul = base + NA_OFF_MAPMUL;
    int *src = (int *)(base + NA_OFF_MAPSRC);
    BcMap mp, mw;
    mp.x = {src + 0 * NOALLOC_AXIS_LEN, mul + 0 * NOALLOC_AXIS_LEN};
    mp.y = {src + 1 * NOALLOC_AXIS_LEN, mul + 1 * NOALLOC_AXIS_LEN};
    mw.x = {src + 2 * NOALLOC_AXIS_LEN, mul + 2 * NOALLOC_AXIS_LEN};
    mw.y = {src + 3 * NOALLOC_AXIS_LEN, mul + 3 * NOALLOC_AXIS_LEN};

    // tables into the scratch array; the solver's barrier state and status
    // must start at zero (the planes are fully written before they are read)
    build_tables(*grid, NX, NY);
    if (cudaMemcpyAsync(metric, g_tab.metric, sizeof(g_tab.metric), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(mul, g_tab.mul, sizeof(g_tab.mul), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(src, g_tab.src, sizeof(g_tab.src), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(base + NA_OFF_SCAL, 0, sizeof(DevScalars), st) != cudaSuccess)
        return na_err(PVOF_ECUDA, "scratch set-up copy failed");

    const size_t origin = (size_t)NG * d.P + NG;
    double *plane[NA_PLANES];
    for (size_t q = 0; q < NA_PLANES; q++) plane[q] = base + q * NOALLOC_PLANE_MAX + origin;
    DevScalars *scal = (DevScalars *)(base + NA_OFF_SCAL);

    // Pressure_compute_preconditioner (psolve_cg.c:63-101)
    dim3 blk(32, 8), grd((unsigned)((NX - 1 + 31) / 32), (unsigned)((NY - 1 + 7) / 8));
    k_p_precond<<<grd, blk, 0, st>>>(d, 0, NX - 1, 0, NY - 1, rho + origin, plane[0]);
    if (cudaGetLastError() != cudaSuccess) return na_err(PVOF_ECUDA, "preconditioner launch failed");

    // Pressure_solve_cg (psolve_cg.c:130-293)
    PresArgs A;
    A.d = d;
    A.mp = mp;
    A.phi = phi + origin;
    A.rhs = rhs + origin;
    A.rho = rho + origin;
    A.M = plane[0];
    A.res = plane[1];
    A.dir = plane[2];
    A.dir2 = plane[3];
    A.z = plane[4];
    A.Ad = plane[5];
    A.tol = params->P_CG_ETOL;
    A.maxit = params->P_CG_MAXIT;
    A.partials = base + NA_OFF_PART;
    A.scal = scal;
    const int n = (NX - 1) * (NY - 1);
    int nb = (n + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
    if (nb > sc.coop_blocks) nb = sc.coop_blocks;
    void *args[] = {&A};
    if (cudaLaunchCooperativeKernel((const void *)k_cg_pressure, dim3((unsigned)nb), dim3(NOALLOC_THREADS), args, 0, st) !=
        cudaSuccess)
        return na_err(PVOF_ECUDA, "solver launch failed");

    // exchange of the correction's ghosts after the solve (psolve_cg.c:281-283)
    int nf = 8 * (NY + 2 * NG) + 8 * (NX + 2 * NG);
    k_fill<<<(nf + 255) / 256, 256, 0, st>>>(d, mw, phi + origin);
    if (cudaGetLastError() != cudaSuccess) return na_err(PVOF_ECUDA, "ghost update launch failed");

    DevScalars h;
    if (cudaMemcpyAsync(&h, scal, sizeof(DevScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return na_err(PVOF_ECUDA, "solver failed");
    if (h.error) return na_err(PVOF_ECUDA, "solver grid barrier timed out");
    if (iterations) *iterations = h.p_iters;
    if (residual) *residual = h.p_res;
    return h.p_iters;
}
