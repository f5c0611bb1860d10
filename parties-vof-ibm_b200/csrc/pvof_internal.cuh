// Internal definitions of the B200 two-phase substep library.
//
// Device layout: one k plane per field (the 2D modes of PARTIES keep all
// planes identical), stored row-major with a pitch of P doubles.  The pointer
// handed to kernels addresses element (i=0, j=0); element (i,j) is at
// f[j*P + i] for i in [-3, NX+3), j in [-3, NY+3) -- the reference's own
// ghosted index space (PARTIES/src/Memory.c:36-89), so every kernel runs on
// the reference's index ranges.  NX = NXM+1 and NY = NYM+1 include the half
// cell the reference adds at the far end of each direction.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pvof.h"

namespace pvof3 {
struct Handle;
}

namespace pvof {

constexpr int NG = 3;        // ghost layers
constexpr int OX = 4;        // column of i = 0 inside a row (i = -3 at column 1)
constexpr int OY = NG;       // row of j = 0

// RK3 coefficients (PARTIES/src/Include/definitions.h:197-204)
__host__ __device__ inline double bet(int s) { return s == 0 ? 4.0 / 15.0 : (s == 1 ? 1.0 / 15.0 : 1.0 / 6.0); }
__host__ __device__ inline double bet2(int s) { return s == 0 ? 8.0 / 15.0 : (s == 1 ? 2.0 / 15.0 : 1.0 / 3.0); }
__host__ __device__ inline double gamb(int s) { return s == 0 ? 2.0 : (s == 1 ? 25.0 / 4.0 : 9.0 / 2.0); }
__host__ __device__ inline double zetb(int s) { return s == 0 ? 0.0 : (s == 1 ? -17.0 / 4.0 : -2.5); }

// Ghost-update kinds.  Each is the composition of the reference's boundary
// routine and its periodic exchange for one kind of field.
enum BcKind {
    BK_SCALAR = 0,   // VOF_DIFFUSE_set_boundary_values (VOF_DIFFUSE.c:571-683)
    BK_PRESSURE,     // Pressure_apply_BCs + exchange (psolve_cg.c:358-529)
    BK_U,            // Velocity_update_boundaries('u', VEL_TYPE_NORMAL)
    BK_V,            // Velocity_update_boundaries('v', VEL_TYPE_NORMAL)
    BK_U_CG,         // Velocity_update_boundaries('u', VEL_TYPE_CG)
    BK_V_CG,         // Velocity_update_boundaries('v', VEL_TYPE_CG)
    BK_WRAP_C,       // exchange only, scalar component (Communication.c:146-291)
    BK_WRAP_U,       // exchange only, x-face component (U_VELOCITY, FLUX_X)
    BK_WRAP_V,       // exchange only, y-face component (V_VELOCITY, FLUX_Y)
    BK_NRM_X,        // contact-line solid normal, x component (VOF_IBM_wetting.c:914-1016)
    BK_NRM_Y,        // same, y component
    BK_COUNT
};

// Per-axis source maps of one kind: entry [i + NG] for i in [-NG, N + NG).
// src == i and mul == 1 means "not written"; mul == 0 means "set to zero".
struct AxisMap {
    const int *src;
    const double *mul;
};

struct BcMap {
    AxisMap x, y;
};

// Grid metrics, each offset so that m[i] is valid for i in [-NG, N + NG - 1).
struct Metrics {
    const double *idx_u, *idx_c, *dx_c, *dx_u;
    const double *idy_v, *idy_c, *dy_c, *dy_v;
    const double *r_u, *r_c, *inv_r_u, *inv_r_c, *ring_wt_c;
    // inner-product weights of the physical cells: the measure of the cell
    // plus the measures of the G-range half cells that copy it (x: times the
    // ring weight in the axisymmetric mode); cell weight = wx[i] * wy[j] * wz
    const double *wx, *wy;
};

struct Dom {
    int NX, NY;       // G-range extents (NXM+1, NYM+1)
    int P;            // pitch in doubles
    int planar;       // TWOD_CARTESIAN
    int axisym;       // AXISYM_RZ
    int perx, pery;   // XPERIODIC, YPERIODIC
    int nk;           // planes of the reference's G range in k (2 in 2D)
    double slab;      // dummy_z_slab_thickness
    double wz;        // slab (planar) or 1 (axisymmetric) in the cell weights
    Metrics m;
};

__host__ __device__ inline size_t at(const Dom &d, int i, int j) { return (size_t)((ptrdiff_t)j * d.P + i); }

// scratch arrays beyond the public fields
enum Scratch {
    SC_PSI = 0, SC_BULK_S, SC_CH_AUX1, SC_CH_RHS_NM1, SC_CH_RES, SC_CH_DIR, SC_CH_DIR2,
    SC_P_RES, SC_P_D, SC_P_AD, SC_P_MINV,
    SC_U_R, SC_U_D, SC_U_AD, SC_U_DIAG, SC_V_R, SC_V_D, SC_V_AD, SC_V_DIAG,
    SC_OLD, SC_U_D2, SC_V_D2, SC_P_D2, SC_U_Z, SC_V_Z, SC_P_Z, SC_SNAP, SC_PHI_PREV, SC_PHI_PREV1, SC_PHI_PREV2, SC_PHI_OLD, SC_PHI_OLD1, SC_PHI_OLD2, SC_P_HAT,
    SC_P_BX, SC_P_BY, SC_U_FT, SC_U_MC, SC_V_FT, SC_V_MC,
    SC_COUNT
};

// device-side scalars written by solver kernels and read once per substep
struct DevScalars {
    int ch_iters;
    double ch_rel;
    int vel_iters[2];
    double vel_rms[2];
    int p_iters;
    double p_res;
    double div_max;
    double clamp_delta;
    double cnn_ms[2];   // mean squares of the network's rhs and phi_prev inputs
    double mass;
    int error;          // non-zero: a grid barrier gave up (see pvof_cg.cu)
    unsigned bar_count; // grid barrier state
    unsigned bar_gen;
    unsigned long long bar_arrivals;   // arrivals at the counting grid barrier, zeroed before each launch
};

// launch shape of a strip solver: threads per CTA (0: the range does not fit)
// and dynamic shared memory
struct StripPlan {
    size_t smem;
    int threads;
};

struct IbmState;

// host state that the launches of a substep (up to its first Poisson pass)
// depend on, the key of its captured CUDA graph
struct GraphKey {
    int stage;
    double dt;
    const double *fsig;   // the f_sigma buffers swap every substep
    int warm, one_cluster;
};

struct GraphEntry {
    GraphKey key;
    int state;   // 0 empty, 1 seen once, 2 captured, 3 runs directly
    cudaGraphExec_t exec;
    long long launches;   // kernels in the graph
};

struct Ctx {
    pvof_grid_desc g;
    pvof_params p;
    int device;
    Dom dom;
    size_t plane_elems;      // P * (NY + 2*NG)
    double *base[PVOF_F_COUNT];   // allocation bases
    double *f[PVOF_F_COUNT];      // element (0,0) of each field
    double *sbase[SC_COUNT];
    double *s[SC_COUNT];
    double *metric_mem;
    int *map_src_mem;
    double *map_mul_mem;
    BcMap maps[BK_COUNT];
    double *partials;        // per-block partial sums (3 per block)
    DevScalars *scal;        // device scalars
    DevScalars *scal_host;   // pinned host mirror
    double *host_plane;      // pinned staging plane for uploads/downloads
    cudaStream_t stream;
    int stage;
    double dt;
    double time;
    double clamp_total;      // clamp_mass summed over the substeps since pvof_initialize
    size_t cgs_p_smem;       // shared memory of the cluster pressure solver (0: grid solver)
    size_t cgs_v_smem;       // same, velocity solver for both components (0: grid solver)
    int cgs_p_threads, cgs_v_threads;   // their threads per CTA
    StripPlan cgs_p_fit, cgs_v_fit;     // the cluster plans that fit this grid (kept for pvof_set_cluster_solvers)
    int vel_one_cluster;     // momentum solve as u then v on one cluster (batched runs)
    int pressure_pairs;      // grid-wide pressure solve over pairs of cells: -1 by size, 0 never, 1 always
    int phi_prev_mask;       // stages whose last correction is kept in SC_PHI_PREV + stage
    int phi_old_mask;        // stages whose correction one step before that is in SC_PHI_OLD + stage
    // learned warm start (pvof_cnn.cu): FP32 and BF16 parameters, the input
    // planes, the output plane and the activations
    float *cnn_params;
    uint16_t *cnn_bf16;
    float *cnn_x, *cnn_y, *cnn_work;
    int coop_blocks;         // the most co-resident blocks of any grid-wide solver (sizes the partial sums)
    int coop_blocks_of[3];   // co-resident blocks of each grid-wide solver, by PVOF_SOLVER_*
    int coop_threads;
    long long launches;      // kernels launched by this context
    // measurement
    cudaEvent_t timer_ev[2];
    double *flush_buf;
    double *host_stage;      // contiguous staging of one field block for the host copies
    size_t host_stage_elems;
    size_t flush_bytes;
    int solver_timing;
    static constexpr int NPEND = 16;
    cudaEvent_t pend_ev[NPEND][2];
    int pend_kind[NPEND], pend_comp[NPEND];
    long long pend_cells[NPEND], pend_cells2[NPEND];
    int npend;
    IbmState *ibm;           // resolved particles (null until pvof_set_particles)
    pvof3::Handle *h3;       // the 3D mode's state (PVOF_GEOM_3D); null for the 2D modes
    double *fft_coef;        // as, ap, an (NY-1 each) and the modified wavenumbers (NX-1)
    double *spec_mem;        // spectral pressure preconditioner: twiddles, block sums, reduction tables
    struct SpecScal *spec_s; // its grid barrier state
    double spec_fscale;      // dy^2 / N
    int spec_blocks;         // blocks of its cooperative launch
    double sol_ms[3];
    long long sol_launches[3], sol_iters[3], sol_cell_iters[3];
    int use_graphs;          // replay each substep's launches from a captured CUDA graph
    static constexpr int NGRAPHS = 24;   // 3 stages x 2 buffer parities x warm start x one or two clusters
    GraphEntry graphs[NGRAPHS];
    int graph_next;
    long long graph_replays; // substeps whose launches came from a graph
    struct TuneState *tune;  // stencil tile autotuner (null until pvof_set_autotune)
    struct AdvectMaps *adv_maps;   // tensor maps of the C_L, u, v planes for the advection tiles
};

}  // namespace pvof
