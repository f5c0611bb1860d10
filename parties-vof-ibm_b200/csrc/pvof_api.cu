// C ABI (include/pvof.h) and host orchestration of the two-phase substep.
//
// Each pvof_* routine issues, on the context's stream, the kernels that
// restate one reference routine, in the reference's order, including every
// ghost update the reference performs at that point (file:line citations are
// relative to PARTIES/src).  Nothing here computes on the host; there is no
// CPU fallback: without a CUDA device pvof_create fails with PVOF_ENODEV.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pvof_particles.cuh"
#include "pvof_3d_api.h"

using namespace pvof;

struct pvof_ctx : public Ctx {};

namespace {

thread_local std::string g_err;

int set_err(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_err(PVOF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

#define CKL(ctx)                                                                              \
    do {                                                                                      \
        (ctx)->launches++;                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                  \
        if (e_ != cudaSuccess) return set_err(PVOF_ECUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

#define TRY(x)                      \
    do {                            \
        int rc_ = (x);              \
        if (rc_ < 0) return rc_;    \
    } while (0)

constexpr int TBX = 32, TBY = 8;
constexpr int COOP_THREADS = 512;

bool is_ng(int field)
{
    return (field >= PVOF_F_U_EXPLICIT && field <= PVOF_F_FSIG_NEW_Y) || (field >= PVOF_F_W_EXPLICIT && field <= PVOF_F_FSIG_NEW_Z);
}

// a 3D-mode result: the message of a failure comes from pvof_3d.cu
int from3(int rc)
{
    if (rc < 0) g_err = pvof3::last_error();
    return rc;
}

// ---------------------------------------------------------------------------
// metrics and ghost maps, built on the host exactly as the reference does
// ---------------------------------------------------------------------------

// Grid.c:797-862 (uniform coordinates), :372-420 (widths), :871-918 (radii)
struct HostMetrics {
    std::vector<double> xu, xc, dx_u, dx_c, idx_u, idx_c, yv, yc, dy_v, dy_c, idy_v, idy_c;
    std::vector<double> r_u, r_c, inv_r_u, inv_r_c, ring_wt_c;
    std::vector<double> wx, wy;
};

void build_metrics(const pvof_grid_desc &g, int NX, int NY, HostMetrics &h)
{
    const bool perx = g.periodic[0] != 0, pery = g.periodic[1] != 0;
    int nx = NX + 2 * NG, ny = NY + 2 * NG;
    auto z = [](std::vector<double> &v, int n) { v.assign((size_t)n, 0.0); };
    z(h.xu, nx); z(h.xc, nx); z(h.dx_u, nx); z(h.dx_c, nx); z(h.idx_u, nx); z(h.idx_c, nx);
    z(h.yv, ny); z(h.yc, ny); z(h.dy_v, ny); z(h.dy_c, ny); z(h.idy_v, ny); z(h.idy_c, ny);
    z(h.r_u, nx); z(h.r_c, nx); z(h.inv_r_u, nx); z(h.inv_r_c, nx); z(h.ring_wt_c, nx);
    double Lx = g.xmax - g.xmin, Ly = g.ymax - g.ymin;
    double dx = Lx / (double)(NX - 1), dy = Ly / (double)(NY - 1);
    for (int i = -NG; i < NX + NG; i++) {
        h.xu[i + NG] = g.xmin + i * dx;
        h.xc[i + NG] = g.xmin + (0.5 + i) * dx;
    }
    for (int j = -NG; j < NY + NG; j++) {
        h.yv[j + NG] = g.ymin + j * dy;
        h.yc[j + NG] = g.ymin + (0.5 + j) * dy;
    }
    for (int i = -NG; i < NX + NG - 1; i++) {
        h.dx_u[i + NG] = h.xu[i + 1 + NG] - h.xu[i + NG];
        h.dx_c[i + NG] = h.xc[i + 1 + NG] - h.xc[i + NG];
        h.idx_u[i + NG] = 1.0 / h.dx_u[i + NG];
        h.idx_c[i + NG] = 1.0 / h.dx_c[i + NG];
    }
    for (int j = -NG; j < NY + NG - 1; j++) {
        h.dy_v[j + NG] = h.yv[j + 1 + NG] - h.yv[j + NG];
        h.dy_c[j + NG] = h.yc[j + 1 + NG] - h.yc[j + NG];
        h.idy_v[j + NG] = 1.0 / h.dy_v[j + NG];
        h.idy_c[j + NG] = 1.0 / h.dy_c[j + NG];
    }
    if (g.geometry == PVOF_GEOM_AXISYM) {
        for (int i = -NG; i < NX + NG; i++) {
            double ru = std::fabs(h.xu[i + NG]), rc = std::fabs(h.xc[i + NG]);
            h.r_u[i + NG] = ru;
            h.r_c[i + NG] = rc;
            h.inv_r_u[i + NG] = (ru > 1.0e-14) ? 1.0 / ru : 0.0;
            h.inv_r_c[i + NG] = (rc > 1.0e-14) ? 1.0 / rc : 0.0;
            h.ring_wt_c[i + NG] = g.theta_span * rc;
        }
    }
    // inner-product weights: each G-range position adds its measure to the
    // physical cell the scalar ghost update copies into it (the half cell
    // i = NX-1 copies cell 0 when periodic, NX-2 at a wall; likewise in y)
    h.wx.assign((size_t)nx, 0.0);
    h.wy.assign((size_t)ny, 0.0);
    for (int i = 0; i < NX; i++) {
        int s = (i == NX - 1) ? (perx ? 0 : NX - 2) : i;
        double w = h.dx_u[i + NG];
        if (g.geometry == PVOF_GEOM_AXISYM) w = w * h.ring_wt_c[i + NG];
        h.wx[s + NG] += w;
    }
    for (int j = 0; j < NY; j++) {
        int s = (j == NY - 1) ? (pery ? 0 : NY - 2) : j;
        h.wy[s + NG] += h.dy_v[j + NG];
    }
}

struct Map1 {
    std::vector<int> src;
    std::vector<double> mul;
    int N;
    void init(int n)
    {
        N = n;
        src.resize((size_t)n + 2 * NG);
        mul.assign((size_t)n + 2 * NG, 1.0);
        for (int i = -NG; i < n + NG; i++) src[i + NG] = i;
    }
    void set(int i, int s, double m) { src[i + NG] = s; mul[i + NG] = m; }
    // scalar-component periodic exchange (Communication.c:168-229)
    void wrap_scalar()
    {
        for (int i = -NG; i <= -1; i++) set(i, i + (N - 1), 1.0);
        for (int i = N - 1; i <= N + 1; i++) set(i, i - (N - 1), 1.0);
    }
    // face-component periodic exchange: first face aliased to the last
    void wrap_face()
    {
        for (int i = -NG; i <= 0; i++) set(i, i + (N - 1), 1.0);
        for (int i = N; i <= N + 2; i++) set(i, i - (N - 1), 1.0);
    }
};

// One axis of one ghost-update kind.  `normal` is true for the velocity
// component normal to this axis' walls (u on x, v on y).
void axis_map(Map1 &m, int kind, int N, bool periodic, int wall_lo, int wall_hi, bool axisym_lo, bool normal_u_x,
              bool is_x)
{
    m.init(N);
    bool is_u = (kind == BK_U || kind == BK_U_CG);
    bool is_v = (kind == BK_V || kind == BK_V_CG);
    bool cg = (kind == BK_U_CG || kind == BK_V_CG);
    bool normal = (is_x && is_u) || (!is_x && is_v);
    (void)normal_u_x;
    if (periodic) {
        bool face = (kind == BK_WRAP_U && is_x) || (kind == BK_WRAP_V && !is_x) || (normal && (is_u || is_v));
        if (face) m.wrap_face();
        else m.wrap_scalar();
        return;
    }
    switch (kind) {
    case BK_SCALAR:  // VOF_DIFFUSE.c:591-663
        for (int g = 1; g <= NG; g++) {
            if (axisym_lo) m.set(-g, 0, 1.0);
            else if (wall_lo == PVOF_WALL_FREESLIP) m.set(-g, g - 1, 1.0);
            else m.set(-g, 0, 1.0);
        }
        for (int g = 0; g < NG; g++) {
            if (wall_hi == PVOF_WALL_FREESLIP) m.set(N - 1 + g, N - 2 - g, 1.0);
            else m.set(N - 1 + g, N - 2, 1.0);
        }
        break;
    case BK_PRESSURE:  // psolve_cg.c:374-460
        m.set(-1, 0, 1.0);
        m.set(N - 1, N - 2, 1.0);
        break;
    case BK_U:
    case BK_V:
    case BK_U_CG:
    case BK_V_CG:  // Velocity.c:2480-2700
        if (normal) {
            if (!cg || axisym_lo) m.set(0, 0, 0.0);
            if (!cg) m.set(N - 1, N - 1, 0.0);
        } else {
            if (axisym_lo) m.set(-1, 0, 1.0);
            else m.set(-1, 0, wall_lo == PVOF_WALL_NOSLIP ? -1.0 : 1.0);
            m.set(N - 1, N - 2, wall_hi == PVOF_WALL_NOSLIP ? -1.0 : 1.0);
        }
        break;
    case BK_NRM_X:
    case BK_NRM_Y: {  // mcl_apply_normal_parity (VOF_IBM_wetting.c:914-1016), planar mode
        // mirrored across a free-slip wall; the component normal to the wall flips
        const double sgn = ((kind == BK_NRM_X) == is_x) ? -1.0 : 1.0;
        if (wall_lo == PVOF_WALL_FREESLIP && !axisym_lo)
            for (int g = 1; g <= NG; g++) m.set(-g, g - 1, sgn);
        if (wall_hi == PVOF_WALL_FREESLIP)
            for (int g = 0; g < NG; g++) m.set(N - 1 + g, N - 2 - g, sgn);
        break;
    }
    default:  // exchange-only kinds on a walled axis: nothing
        break;
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
// --- stencil tile autotuner -----------------------------------------------
// The cell-wise kernels issued through launch2d compute every cell with the
// same arithmetic whatever the thread-block shape, so their tile is free.
// pvof_set_autotune starts an online tuning over the context's next
// substeps: each launch of a tunable kernel takes the candidate tile with
// the fewest samples so far, bracketed by events; after every candidate has
// TUNE_SAMPLES samples the kernel keeps the tile of the smallest mean time.
// While tuning, substeps run launch by launch (no graph capture); the
// results are bit for bit those of the default tile.
struct Tile {
    int bx, by;
};
constexpr Tile TUNE_TILES[] = {{TBX, TBY}, {64, 4}, {128, 2}, {256, 1}, {32, 4}, {64, 8}};
constexpr int NTILES = sizeof(TUNE_TILES) / sizeof(TUNE_TILES[0]);
constexpr int TUNE_SAMPLES = 2;
constexpr int TUNE_EVENTS = 64;

struct TuneRec {
    const void *fn;
    const char *name;
    double ms[NTILES];
    int n[NTILES];
    int chosen;   // index into TUNE_TILES, -1 while undecided
};

}  // namespace

struct pvof::TuneState {
    bool active = false;
    std::vector<TuneRec> recs;
    cudaEvent_t ev[TUNE_EVENTS][2];
    int pend_rec[TUNE_EVENTS], pend_tile[TUNE_EVENTS];
    int npend = 0;
    bool events = false;
    ~TuneState()
    {
        if (events)
            for (int q = 0; q < TUNE_EVENTS; q++) {
                cudaEventDestroy(ev[q][0]);
                cudaEventDestroy(ev[q][1]);
            }
    }
};

namespace {

// the kernels the autotuner may retile (cell-wise, no block-level reductions)
const TuneRec *tunable(const void *fn)
{
    static const std::vector<TuneRec> table = [] {
        std::vector<TuneRec> t;
        auto add = [&](const void *fn, const char *name) {
            TuneRec r;
            std::memset(&r, 0, sizeof(r));
            r.fn = fn;
            r.name = name;
            r.chosen = -1;
            t.push_back(r);
        };
#define PVOF_TUNABLE(k) add((const void *)k, #k)
        PVOF_TUNABLE(k_laplacian); PVOF_TUNABLE(k_laplacian_f); PVOF_TUNABLE(k_bulk_S); PVOF_TUNABLE(k_bulk_S_f);
        PVOF_TUNABLE(k_psi_LG); PVOF_TUNABLE(k_psi_LG_f); PVOF_TUNABLE(k_f_sigma); PVOF_TUNABLE(k_f_sigma_f);
        PVOF_TUNABLE(k_u_impexp); PVOF_TUNABLE(k_v_impexp); PVOF_TUNABLE(k_set_rhs); PVOF_TUNABLE(k_rhs_vec);
        PVOF_TUNABLE(k_p_rhs); PVOF_TUNABLE(k_p_precond); PVOF_TUNABLE(k_p_update); PVOF_TUNABLE(k_project);
        PVOF_TUNABLE(k_density); PVOF_TUNABLE(k_cell_center); PVOF_TUNABLE(k_gravity); PVOF_TUNABLE(k_add);
        PVOF_TUNABLE(k_add_to); PVOF_TUNABLE(k_sub_scaled); PVOF_TUNABLE(k_div_by);
#undef PVOF_TUNABLE
        return t;
    }();
    for (const TuneRec &r : table)
        if (r.fn == fn) return &r;
    return nullptr;
}

// the tile of a launch; with the tuner active, a candidate and an event slot
// (slot >= 0: record ev[slot][1] after the launch)
Tile tune_pick(pvof_ctx *c, const void *fn, int &slot)
{
    slot = -1;
    TuneState *t = c->tune;
    if (!t) return TUNE_TILES[0];
    int q = -1;
    for (size_t k = 0; k < t->recs.size(); k++)
        if (t->recs[k].fn == fn) { q = (int)k; break; }
    if (q < 0) {
        const TuneRec *r = tunable(fn);
        if (!r) return TUNE_TILES[0];
        t->recs.push_back(*r);
        q = (int)t->recs.size() - 1;
    }
    TuneRec &r = t->recs[(size_t)q];
    if (r.chosen >= 0) return TUNE_TILES[r.chosen];
    if (!t->active || !t->events || t->npend >= TUNE_EVENTS) return TUNE_TILES[0];
    int best = 0;
    for (int k = 1; k < NTILES; k++)
        if (r.n[k] < r.n[best]) best = k;
    slot = t->npend++;
    t->pend_rec[slot] = q;
    t->pend_tile[slot] = best;
    if (cudaEventRecord(t->ev[slot][0], c->stream) != cudaSuccess) {
        t->npend--;
        slot = -1;
        return TUNE_TILES[0];
    }
    return TUNE_TILES[best];
}

// after a stream synchronisation: the finished samples into their kernels,
// decisions for the kernels with every candidate sampled; the tuner stops
// when every kernel seen so far is decided
void collect_tune(pvof_ctx *c)
{
    TuneState *t = c->tune;
    if (!t || !t->active) return;
    for (int q = 0; q < t->npend; q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t->ev[q][0], t->ev[q][1]) != cudaSuccess) continue;
        TuneRec &r = t->recs[(size_t)t->pend_rec[q]];
        r.ms[t->pend_tile[q]] += ms;
        r.n[t->pend_tile[q]] += 1;
    }
    t->npend = 0;
    bool all = !t->recs.empty();
    for (TuneRec &r : t->recs) {
        if (r.chosen >= 0) continue;
        bool done = true;
        for (int k = 0; k < NTILES; k++) done = done && r.n[k] >= TUNE_SAMPLES;
        if (!done) { all = false; continue; }
        int best = 0;
        for (int k = 1; k < NTILES; k++)
            if (r.ms[k] / r.n[k] < r.ms[best] / r.n[best]) best = k;
        r.chosen = best;
    }
    if (all) t->active = false;
}

template <class K, class... Args>
int launch2d(pvof_ctx *c, K kernel, int i0, int i1, int j0, int j1, Args... args)
{
    if (i1 <= i0 || j1 <= j0) return PVOF_OK;
    int slot;
    const Tile t = tune_pick(c, (const void *)kernel, slot);
    dim3 blk((unsigned)t.bx, (unsigned)t.by);
    dim3 grd((unsigned)((i1 - i0 + t.bx - 1) / t.bx), (unsigned)((j1 - j0 + t.by - 1) / t.by));
    kernel<<<grd, blk, 0, c->stream>>>(c->dom, i0, i1, j0, j1, args...);
    CKL(c);
    if (slot >= 0) CK(cudaEventRecord(c->tune->ev[slot][1], c->stream));
    return PVOF_OK;
}

int fill(pvof_ctx *c, int kind, double *f)
{
    int n = 8 * (c->dom.NY + 2 * NG) + 8 * (c->dom.NX + 2 * NG);
    k_fill<<<(n + 255) / 256, 256, 0, c->stream>>>(c->dom, c->maps[kind], f);
    CKL(c);
    return PVOF_OK;
}

// blocks for a grid-wide solver launch of kind PVOF_SOLVER_*: enough for n
// cells, at most what that kernel keeps co-resident
int coop_blocks(pvof_ctx *c, int n, int kind)
{
    int b = (n + COOP_THREADS - 1) / COOP_THREADS;
    if (b > c->coop_blocks_of[kind]) b = c->coop_blocks_of[kind];
    if (b < 1) b = 1;
    return b;
}

// Issue one solver launch, bracketed by timing events when enabled.
// kind: PVOF_SOLVER_*; comp: velocity component (0/1); n: cells solved.
template <class L>
int timed_launch(pvof_ctx *c, int kind, int comp, int n, L launch, int n2 = 0)
{
    int slot = -1;
    if (c->solver_timing && c->npend < Ctx::NPEND) {
        slot = c->npend++;
        c->pend_kind[slot] = kind;
        c->pend_comp[slot] = comp;
        c->pend_cells[slot] = n;
        c->pend_cells2[slot] = n2;
        CK(cudaEventRecord(c->pend_ev[slot][0], c->stream));
    }
    CK(launch());
    c->launches++;
    if (slot >= 0) CK(cudaEventRecord(c->pend_ev[slot][1], c->stream));
    return PVOF_OK;
}

template <class A>
int coop_launch(pvof_ctx *c, const void *fn, A &args, int n, int kind, int comp)
{
    int nb = coop_blocks(c, n, kind);
    // the solvers' counting grid barriers start from zero arrivals
    CK(cudaMemsetAsync(&c->scal->bar_arrivals, 0, sizeof(unsigned long long), c->stream));
    return timed_launch(c, kind, comp, n, [&]() {
        void *params[] = {&args};
        return cudaLaunchCooperativeKernel(fn, dim3((unsigned)nb), dim3(COOP_THREADS), params, 0, c->stream);
    });
}

// after a stream synchronisation: fold the finished solver launches into the
// per-solver totals (iteration counts come from the device scalars)
void collect_solver_timing(pvof_ctx *c)
{
    const DevScalars &h = *c->scal_host;
    for (int q = 0; q < c->npend; q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c->pend_ev[q][0], c->pend_ev[q][1]) != cudaSuccess) continue;
        int k = c->pend_kind[q], comp = c->pend_comp[q];
        c->sol_ms[k] += ms;
        c->sol_launches[k] += 1;
        if (k == PVOF_SOLVER_VELOCITY && comp == 2) {   // both components in one launch
            c->sol_iters[k] += (long long)h.vel_iters[0] + h.vel_iters[1];
            c->sol_cell_iters[k] += h.vel_iters[0] * c->pend_cells[q] + h.vel_iters[1] * c->pend_cells2[q];
            continue;
        }
        long long it = k == PVOF_SOLVER_BIHARMONIC ? h.ch_iters : (k == PVOF_SOLVER_VELOCITY ? h.vel_iters[comp] : h.p_iters);
        c->sol_iters[k] += it;
        c->sol_cell_iters[k] += it * c->pend_cells[q];
    }
    c->npend = 0;
}

double *F(pvof_ctx *c, int id) { return c->f[id]; }
// resolved solid particles on (the reference's VOF_IBM and LAG_PARTICLE_RESOLVED
// builds): from the first pvof_set_particles call on, even with no particles
int resolved(const pvof_ctx *c) { return c->ibm != nullptr; }
double *S(pvof_ctx *c, int id) { return c->s[id]; }

// loop ranges of the face-centred arrays (e.g. Velocity.c:395-410)
void u_range(const pvof_ctx *c, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 1; i1 = c->dom.NX - 1; j0 = 0; j1 = c->dom.NY - 1;
    if (c->dom.perx) i1 = c->dom.NX;
}
void v_range(const pvof_ctx *c, int &i0, int &i1, int &j0, int &j1)
{
    i0 = 0; i1 = c->dom.NX - 1; j0 = 1; j1 = c->dom.NY - 1;
    if (c->dom.pery) j1 = c->dom.NY;
}

// ---------------------------------------------------------------------------
// routines
// ---------------------------------------------------------------------------

// the FP32 stencil form: WENO5, chemical-potential and surface-tension
// stencils in single precision (fields, reductions and solvers stay FP64)
bool fp32_stencils(const pvof_ctx *c) { return c->p.stencil_fp32 != 0; }

// VOF_DIFFUSE_compute_laplacian (VOF_DIFFUSE.c:834-861); fp32: the
// single-precision stencil of the FP32 form
int compute_laplacian(pvof_ctx *c, double *in, double *out, bool fp32 = false)
{
    TRY(fill(c, BK_SCALAR, in));
    if (fp32) TRY(launch2d(c, k_laplacian_f, 0, c->dom.NX, 0, c->dom.NY, (const double *)in, out));
    else TRY(launch2d(c, k_laplacian, 0, c->dom.NX, 0, c->dom.NY, (const double *)in, out));
    return fill(c, BK_SCALAR, out);
}

// VOF_DIFFUSE_advect_WENO5 (VOF_DIFFUSE.c:931-996): the face fluxes, their
// ghost update and the divergence in one TMA-tiled kernel (pvof_advect.cu)
int advect(pvof_ctx *c, double *out)
{
    double *CL = F(c, PVOF_F_C_L);
    TRY(fill(c, BK_SCALAR, CL));
    if (!c->adv_maps) {
        c->adv_maps = advect_maps_create(c->base[PVOF_F_C_L], c->base[PVOF_F_U], c->base[PVOF_F_V], c->dom.P, c->dom.NY);
        if (!c->adv_maps) return set_err(PVOF_ECUDA, "cuTensorMapEncodeTiled is not available for the advection tiles");
    }
    CK(advect_tma_launch(c->adv_maps, c->dom, c->maps[BK_WRAP_U], c->maps[BK_WRAP_V], CL, F(c, PVOF_F_U),
                         F(c, PVOF_F_V), c->p.weno_order == 5 ? 1 : 0, fp32_stencils(c) != 0, out, c->scal, c->stream));
    c->launches++;
    return fill(c, BK_SCALAR, out);
}

int phase_cache(pvof_ctx *c)
{
    size_t n = c->plane_elems;
    k_phase_cache<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, c->base[PVOF_F_C_L], c->base[PVOF_F_C_S],
                                                                      c->base[PVOF_F_C_G], c->base[PVOF_F_F]);
    CKL(c);
    return PVOF_OK;
}

int bound(pvof_ctx *c)
{
    const int NX = c->dom.NX, NY = c->dom.NY;
    dim3 blk(TBX, TBY);
    dim3 grd((unsigned)((NX + TBX - 1) / TBX), (unsigned)((NY + TBY - 1) / TBY));
    k_bound<<<grd, blk, 0, c->stream>>>(c->dom, 0, NX, 0, NY, F(c, PVOF_F_C_L), F(c, PVOF_F_C_S), F(c, PVOF_F_C_G),
                                        c->partials);
    CKL(c);
    k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials, (int)(grd.x * grd.y), &c->scal->clamp_delta);
    CKL(c);
    return PVOF_OK;
}

// resolved-particle routines (defined with the particle bookkeeping below)
int compute_C_S(pvof_ctx *c);
int apply_contact_angle(pvof_ctx *c);
int extend_psi_LG(pvof_ctx *c);
int ibm_flag_points(pvof_ctx *c);
int ibm_force(pvof_ctx *c, int force_iter);
int vel_explicit(pvof_ctx *c, int comp);
int ibm_advect(pvof_ctx *c);
int ibm_velocity_init(pvof_ctx *c);

// VOF_DIFFUSE_init (VOF_DIFFUSE.c:523-568)
int vof_diffuse_init(pvof_ctx *c)
{
    if (resolved(c)) TRY(compute_C_S(c));
    size_t n = c->plane_elems;
    k_clamp_from<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, c->base[PVOF_F_F], c->base[PVOF_F_C_L]);
    CKL(c);
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_C_L)));
    TRY(phase_cache(c));
    TRY(bound(c));
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_C_L)));
    TRY(phase_cache(c));
    if (resolved(c)) TRY(apply_contact_angle(c));
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_C_L)));
    TRY(phase_cache(c));
    return fill(c, BK_SCALAR, F(c, PVOF_F_C_G));
}

int vof_diffuse_step(pvof_ctx *c)
{
    const int NX = c->dom.NX, NY = c->dom.NY, s = c->stage;
    const double a_dt = 1.0 / (c->dt * bet(s));
    const double bih = c->p.Cn * c->p.Cn / c->p.Pe_CH;
    double *CL = F(c, PVOF_F_C_L), *cur = F(c, PVOF_F_CH_RHS_CUR), *aux = S(c, SC_CH_AUX1);
    double *vec = S(c, SC_CH_RHS_NM1), *rn = F(c, PVOF_F_CH_RHS_N), *bS = S(c, SC_BULK_S);
    double *psiLG = F(c, PVOF_F_PSI_LG);
    // R(C) = -div(u C) + Pe^-1 L S(C)  (VOF_DIFFUSE.c:1287-1297)
    TRY(advect(c, cur));
    if (fp32_stencils(c)) TRY(launch2d(c, k_bulk_S_f, 0, NX, 0, NY, (const double *)CL, (const double *)F(c, PVOF_F_C_S), bS));
    else TRY(launch2d(c, k_bulk_S, 0, NX, 0, NY, (const double *)CL, (const double *)F(c, PVOF_F_C_S), bS));
    TRY(fill(c, BK_SCALAR, bS));
    TRY(compute_laplacian(c, bS, aux, fp32_stencils(c)));
    TRY(launch2d(c, k_div_by, 0, NX, 0, NY, aux, c->p.Pe_CH));
    TRY(fill(c, BK_SCALAR, aux));
    TRY(launch2d(c, k_add, 0, NX, 0, NY, cur, (const double *)aux));
    TRY(fill(c, BK_SCALAR, cur));
    TRY(launch2d(c, k_rhs_vec, 0, NX, 0, NY, vec, (const double *)CL, (const double *)cur, (const double *)rn, a_dt, s));
    TRY(fill(c, BK_SCALAR, vec));
    // implicit biharmonic (VOF_DIFFUSE.c:1018-1069)
    TRY(compute_laplacian(c, CL, aux));
    TRY(compute_laplacian(c, aux, psiLG));
    TRY(launch2d(c, k_sub_scaled, 0, NX, 0, NY, vec, (const double *)psiLG, bih));
    BihArgs A;
    A.d = c->dom;
    A.msc = c->maps[BK_SCALAR];
    A.x = CL;
    A.b = vec;
    A.r = S(c, SC_CH_RES);
    A.p1 = S(c, SC_CH_DIR);
    A.p2 = S(c, SC_CH_DIR2);
    A.Ap = F(c, PVOF_F_LAP_C);
    A.aux = aux;
    A.a_dt = a_dt;
    A.bih = bih;
    A.tol = (c->p.ch_tol > 0.0) ? c->p.ch_tol : c->p.CG_ETOL;
    A.maxit = (c->p.ch_iter_max > 0) ? c->p.ch_iter_max : c->p.CG_MAXIT;
    A.partials = c->partials;
    A.scal = c->scal;
    TRY(coop_launch(c, (const void *)k_cg_biharmonic, A, NX * NY, PVOF_SOLVER_BIHARMONIC, 0));
    TRY(fill(c, BK_SCALAR, CL));
    // clamp, phase cache, history shift (VOF_DIFFUSE.c:1324-1358)
    TRY(bound(c));
    TRY(fill(c, BK_SCALAR, CL));
    TRY(phase_cache(c));
    if (resolved(c) && s == 2) {
        // contact-angle projection once per time step, then C_L + C_S <= 1
        TRY(apply_contact_angle(c));
        TRY(fill(c, BK_SCALAR, CL));
        TRY(bound(c));
        TRY(fill(c, BK_SCALAR, CL));
        TRY(phase_cache(c));
    }
    size_t bytes = c->plane_elems * sizeof(double);
    CK(cudaMemcpyAsync(c->sbase[SC_CH_RHS_NM1], c->base[PVOF_F_CH_RHS_N], bytes,
                       cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->base[PVOF_F_CH_RHS_N], c->base[PVOF_F_CH_RHS_CUR], bytes, cudaMemcpyDeviceToDevice, c->stream));
    return PVOF_OK;
}

int update_density_viscosity(pvof_ctx *c)
{
    const double rho_g = c->p.rho2 / c->p.rho1, mu_g = c->p.mu2 / c->p.mu1;
    TRY(launch2d(c, k_density, 0, c->dom.NX, 0, c->dom.NY, (const double *)F(c, PVOF_F_C_L),
                 (const double *)F(c, PVOF_F_C_S), (const double *)F(c, PVOF_F_C_G), F(c, PVOF_F_RHO), F(c, PVOF_F_MU),
                 rho_g, mu_g));
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_RHO)));
    return fill(c, BK_SCALAR, F(c, PVOF_F_MU));
}

int compute_psi_LG(pvof_ctx *c)
{
    double *CL = F(c, PVOF_F_C_L), *lap = F(c, PVOF_F_LAP_C), *psi = F(c, PVOF_F_PSI_LG);
    TRY(compute_laplacian(c, CL, lap, fp32_stencils(c)));
    if (fp32_stencils(c))
        TRY(launch2d(c, k_psi_LG_f, 0, c->dom.NX, 0, c->dom.NY, (const double *)CL, (const double *)lap, psi,
                     c->p.Cn * c->p.Cn));
    else
        TRY(launch2d(c, k_psi_LG, 0, c->dom.NX, 0, c->dom.NY, (const double *)CL, (const double *)lap, psi,
                     c->p.Cn * c->p.Cn));
    return fill(c, BK_SCALAR, psi);
}

int compute_f_sigma(pvof_ctx *c)
{
    int ui0, ui1, uj0, uj1, vi0, vi1, vj0, vj1;
    u_range(c, ui0, ui1, uj0, uj1);
    v_range(c, vi0, vi1, vj0, vj1);
    const double scale = 2.0 * 6.0 * std::sqrt(2.0) / (c->p.Cn * c->p.We + 1e-30);
    if (fp32_stencils(c))
        return launch2d(c, k_f_sigma_f, 0, c->dom.NX, 0, c->dom.NY, (const double *)F(c, PVOF_F_C_L),
                        (const double *)F(c, PVOF_F_C_G), (const double *)F(c, PVOF_F_C_S),
                        (const double *)F(c, PVOF_F_PSI_LG), F(c, PVOF_F_FSIG_NEW_X), F(c, PVOF_F_FSIG_NEW_Y), scale,
                        ui0, ui1, uj1, vj0, vi1, vj1);
    return launch2d(c, k_f_sigma, 0, c->dom.NX, 0, c->dom.NY, (const double *)F(c, PVOF_F_C_L),
                    (const double *)F(c, PVOF_F_C_G), (const double *)F(c, PVOF_F_C_S),
                    (const double *)F(c, PVOF_F_PSI_LG), F(c, PVOF_F_FSIG_NEW_X), F(c, PVOF_F_FSIG_NEW_Y), scale, ui0,
                    ui1, uj1, vj0, vi1, vj1);
}

int apply_f_sigma_old(pvof_ctx *c)
{
    int i0, i1, j0, j1;
    u_range(c, i0, i1, j0, j1);
    TRY(launch2d(c, k_add_to, i0, i1, j0, j1, F(c, PVOF_F_U_RHS), (const double *)F(c, PVOF_F_FSIG_OLD_X)));
    v_range(c, i0, i1, j0, j1);
    return launch2d(c, k_add_to, i0, i1, j0, j1, F(c, PVOF_F_V_RHS), (const double *)F(c, PVOF_F_FSIG_OLD_Y));
}

void swap_f_sigma(pvof_ctx *c)
{
    std::swap(c->f[PVOF_F_FSIG_OLD_X], c->f[PVOF_F_FSIG_NEW_X]);
    std::swap(c->base[PVOF_F_FSIG_OLD_X], c->base[PVOF_F_FSIG_NEW_X]);
    std::swap(c->f[PVOF_F_FSIG_OLD_Y], c->f[PVOF_F_FSIG_NEW_Y]);
    std::swap(c->base[PVOF_F_FSIG_OLD_Y], c->base[PVOF_F_FSIG_NEW_Y]);
}

int add_gravity(pvof_ctx *c)
{
    const double *gr = c->p.grav;
    double gm = std::sqrt(gr[0] * gr[0] + gr[1] * gr[1]);
    double gx = 0.0, gy = 0.0;
    if (gm > 0.0) { gx = gr[0] / gm; gy = gr[1] / gm; }
    int i0, i1, j0, j1;
    u_range(c, i0, i1, j0, j1);
    TRY(launch2d(c, k_gravity, i0, i1, j0, j1, (const double *)F(c, PVOF_F_RHO), F(c, PVOF_F_U_RHS), 1, 0,
                 c->p.richardson, gx));
    v_range(c, i0, i1, j0, j1);
    return launch2d(c, k_gravity, i0, i1, j0, j1, (const double *)F(c, PVOF_F_RHO), F(c, PVOF_F_V_RHS), 0, 1,
                    c->p.richardson, gy);
}

int cell_center(pvof_ctx *c)
{
    TRY(fill(c, BK_WRAP_U, F(c, PVOF_F_U)));
    TRY(fill(c, BK_WRAP_V, F(c, PVOF_F_V)));
    return launch2d(c, k_cell_center, -NG, c->dom.NX + NG - 1, -NG, c->dom.NY + NG - 1, (const double *)F(c, PVOF_F_U),
                    (const double *)F(c, PVOF_F_V), F(c, PVOF_F_U_BC), F(c, PVOF_F_V_BC));
}

int implicit_explicit(pvof_ctx *c, int comp)
{
    int i0, i1, j0, j1;
    double iRe = 1.0 / c->p.Re;
    if (comp == 0) {
        u_range(c, i0, i1, j0, j1);
        return launch2d(c, k_u_impexp, i0, i1, j0, j1, (const double *)F(c, PVOF_F_U), (const double *)F(c, PVOF_F_V),
                        (const double *)F(c, PVOF_F_U_BC), (const double *)F(c, PVOF_F_MU), F(c, PVOF_F_U_EXPLICIT),
                        F(c, PVOF_F_U_IMPLICIT), F(c, PVOF_F_U_VISC_EXPLICIT), iRe);
    }
    v_range(c, i0, i1, j0, j1);
    return launch2d(c, k_v_impexp, i0, i1, j0, j1, (const double *)F(c, PVOF_F_U), (const double *)F(c, PVOF_F_V),
                    (const double *)F(c, PVOF_F_V_BC), (const double *)F(c, PVOF_F_MU), F(c, PVOF_F_V_EXPLICIT),
                    F(c, PVOF_F_V_IMPLICIT), F(c, PVOF_F_V_VISC_EXPLICIT), iRe);
}

int set_rhs(pvof_ctx *c, int comp)
{
    int s = c->stage;
    double a_dt = 1.0 / (c->dt * bet(s));
    int i0, i1, j0, j1;
    if (comp == 0) {
        u_range(c, i0, i1, j0, j1);
        return launch2d(c, k_set_rhs, i0, i1, j0, j1, 0, (const double *)F(c, PVOF_F_U), (const double *)F(c, PVOF_F_P),
                        (const double *)F(c, PVOF_F_RHO), F(c, PVOF_F_U_RHS), (const double *)F(c, PVOF_F_U_EXPLICIT),
                        F(c, PVOF_F_U_EXPLICIT_OLD), (const double *)F(c, PVOF_F_U_VISC_EXPLICIT),
                        F(c, PVOF_F_U_VISC_EXPLICIT_OLD), (const double *)F(c, PVOF_F_U_IMPLICIT), a_dt, s,
                        -c->p.dp_dx, resolved(c));
    }
    v_range(c, i0, i1, j0, j1);
    return launch2d(c, k_set_rhs, i0, i1, j0, j1, 1, (const double *)F(c, PVOF_F_V), (const double *)F(c, PVOF_F_P),
                    (const double *)F(c, PVOF_F_RHO), F(c, PVOF_F_V_RHS), (const double *)F(c, PVOF_F_V_EXPLICIT),
                    F(c, PVOF_F_V_EXPLICIT_OLD), (const double *)F(c, PVOF_F_V_VISC_EXPLICIT),
                    F(c, PVOF_F_V_VISC_EXPLICIT_OLD), (const double *)F(c, PVOF_F_V_IMPLICIT), a_dt, s, -c->p.dp_dx,
                    resolved(c));
}

VelArgs vel_args(pvof_ctx *c, int comp)
{
    VelArgs A;
    A.d = c->dom;
    A.comp = comp;
    A.mcg = c->maps[comp == 0 ? BK_U_CG : BK_V_CG];
    if (comp == 0) u_range(c, A.i0, A.i1, A.j0, A.j1);
    else v_range(c, A.i0, A.i1, A.j0, A.j1);
    A.x = F(c, comp == 0 ? PVOF_F_U : PVOF_F_V);
    A.rhs = F(c, comp == 0 ? PVOF_F_U_RHS : PVOF_F_V_RHS);
    A.rho = F(c, PVOF_F_RHO);
    A.mu = F(c, PVOF_F_MU);
    A.r = S(c, comp == 0 ? SC_U_R : SC_V_R);
    A.dir = S(c, comp == 0 ? SC_U_D : SC_V_D);
    A.dir2 = S(c, comp == 0 ? SC_U_D2 : SC_V_D2);
    A.z = S(c, comp == 0 ? SC_U_Z : SC_V_Z);
    A.Ad = S(c, comp == 0 ? SC_U_AD : SC_V_AD);
    A.diag = S(c, comp == 0 ? SC_U_DIAG : SC_V_DIAG);
    A.iRe = 1.0 / c->p.Re;
    A.alpha_dt = bet(c->stage) * c->dt;
    const int NX = c->dom.NX, NY = c->dom.NY, NZ = 2;
    if (comp == 0) A.in_tot = c->dom.perx ? 1.0 / (double)((NX - 1) * (NY - 1) * (NZ - 1)) : 1.0 / (double)((NX - 2) * (NY - 1) * (NZ - 1));
    else A.in_tot = c->dom.pery ? 1.0 / (double)((NX - 1) * (NY - 1) * (NZ - 1)) : 1.0 / (double)((NX - 1) * (NY - 2) * (NZ - 1));
    A.tol = c->p.CG_ETOL;
    // msolve_cg.c's 1e-14 in the step length and the direction update; the
    // unregularised form keeps only a guard against 0 / 0
    A.step_eps = c->p.velocity_cg_unregularized ? 1e-300 : 1e-14;
    A.maxit = c->p.CG_MAXIT;
    A.partials = c->partials;
    A.scal = c->scal;
    A.ft = S(c, comp == 0 ? SC_U_FT : SC_V_FT);
    A.mc = S(c, comp == 0 ? SC_U_MC : SC_V_MC);
    return A;
}

// Velocity_solve_cg (msolve_cg.c:525-722) for one component
int velocity_solve(pvof_ctx *c, int comp)
{
    VelPair V;
    V.c[0] = vel_args(c, comp);
    const int n = (V.c[0].i1 - V.c[0].i0) * (V.c[0].j1 - V.c[0].j0);
    if (c->cgs_v_smem)
        return timed_launch(c, PVOF_SOLVER_VELOCITY, comp, n,
                            [&]() { return cgs_velocity_launch(V, 1, StripPlan{c->cgs_v_smem, c->cgs_v_threads}, c->stream); });
    return coop_launch(c, (const void *)k_cg_velocity, V.c[0], n, PVOF_SOLVER_VELOCITY, comp);
}

// both components: one launch of two clusters when the ranges fit, else in turn
int velocity_solve_both(pvof_ctx *c)
{
    if (!c->cgs_v_smem || c->vel_one_cluster) {
        TRY(velocity_solve(c, 0));
        return velocity_solve(c, 1);
    }
    VelPair V;
    V.c[0] = vel_args(c, 0);
    V.c[1] = vel_args(c, 1);
    const int n0 = (V.c[0].i1 - V.c[0].i0) * (V.c[0].j1 - V.c[0].j0);
    const int n1 = (V.c[1].i1 - V.c[1].i0) * (V.c[1].j1 - V.c[1].j0);
    return timed_launch(c, PVOF_SOLVER_VELOCITY, 2, n0, [&]() { return cgs_velocity_launch(V, 2, StripPlan{c->cgs_v_smem, c->cgs_v_threads}, c->stream); }, n1);
}

}  // namespace

// the host copy of idx_u[1] is needed for the pressure RHS scale
static double host_idx_u1(const pvof_ctx *c)
{
    double Lx = c->g.xmax - c->g.xmin;
    int NX = c->g.NXM + 1;
    double dx = Lx / (double)(NX - 1);
    double xu1 = c->g.xmin + 1 * dx, xu2 = c->g.xmin + 2 * dx;
    return 1.0 / (xu2 - xu1);
}

namespace {

int p_precond(pvof_ctx *c);

// the learned warm start's network inputs (and target) from the density, the
// pressure right-hand side and the kept corrections (pvof_cnn.cu)
int cnn_prepare(pvof_ctx *c, const double *phi_prev, const double *phi, float *x, float *t)
{
    const unsigned nb = 148;
    const int n = (c->dom.NX - 1) * (c->dom.NY - 1);
    double *r0 = S(c, SC_SNAP);   // free during the pressure solve
    k_cnn_residual<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->dom, c->maps[BK_PRESSURE], F(c, PVOF_F_RHO),
                                                                      F(c, PVOF_F_P_RHS), phi_prev, r0);
    CKL(c);
    k_cnn_sumsq<<<nb, 256, 0, c->stream>>>(c->dom, r0, phi_prev, c->partials);
    CKL(c);
    k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials, (int)nb, &c->scal->cnn_ms[0]);
    CKL(c);
    k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials + nb, (int)nb, &c->scal->cnn_ms[1]);
    CKL(c);
    k_cnn_assemble<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->dom, F(c, PVOF_F_RHO), r0, phi_prev, phi,
                                                                      c->scal, x, t);
    CKL(c);
    return PVOF_OK;
}

// warm: start from the correction of the same stage of the previous time
// step instead of zero (the warm-start form); with the network set and
// pressure_warm_start == 2, from that correction plus the network's
// predicted change
int p_set_rhs(pvof_ctx *c, bool warm = false)
{
    double a_dt = 1.0 / (c->dt * 2.0 * bet(c->stage));
    double ihdt = host_idx_u1(c) * a_dt;
    TRY(launch2d(c, k_p_rhs, 0, c->dom.NX - 1, 0, c->dom.NY - 1, (const double *)F(c, PVOF_F_U),
                 (const double *)F(c, PVOF_F_V), F(c, PVOF_F_P_RHS), ihdt));
    if (!warm) {
        CK(cudaMemsetAsync(c->base[PVOF_F_DELTAP], 0, c->plane_elems * sizeof(double), c->stream));
        return PVOF_OK;
    }
    CK(cudaMemcpyAsync(c->base[PVOF_F_DELTAP], c->sbase[SC_PHI_PREV + c->stage], c->plane_elems * sizeof(double),
                       cudaMemcpyDeviceToDevice, c->stream));
    if (c->p.pressure_warm_start == 2 && c->cnn_params) {
        const double *prev = S(c, SC_PHI_PREV + c->stage);
        TRY(cnn_prepare(c, prev, nullptr, c->cnn_x, nullptr));
        const int rc = pvof_cnn_forward(c->cnn_params, c->cnn_bf16, c->cnn_x, c->cnn_y, c->dom.NY - 1, c->dom.NX - 1,
                                        c->cnn_work, c->stream);
        if (rc != PVOF_OK) return set_err(rc, "network forward pass");
        c->launches += 7;
        const int n = (c->dom.NX - 1) * (c->dom.NY - 1);
        const unsigned nb = 148;
        double *e = S(c, SC_P_D2);   // free until the solve starts
        CK(cudaMemsetAsync(c->sbase[SC_P_D2], 0, c->plane_elems * sizeof(double), c->stream));
        k_cnn_expand<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->dom, c->cnn_y, e);
        CKL(c);
        TRY(p_precond(c));   // M for the step; the loop computes it again from the same rho
        k_cnn_galerkin<<<nb, 256, 0, c->stream>>>(c->dom, c->maps[BK_PRESSURE], F(c, PVOF_F_RHO), e, S(c, SC_SNAP),
                                                  S(c, SC_P_MINV), c->partials);
        CKL(c);
        k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials, (int)nb, &c->scal->cnn_ms[0]);
        CKL(c);
        k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials + nb, (int)nb, &c->scal->cnn_ms[1]);
        CKL(c);
        k_cnn_apply<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->dom, e, prev, c->scal, F(c, PVOF_F_DELTAP));
        CKL(c);
    }
    return PVOF_OK;
}

int p_precond(pvof_ctx *c)
{
    return launch2d(c, k_p_precond, 0, c->dom.NX - 1, 0, c->dom.NY - 1, (const double *)F(c, PVOF_F_RHO), S(c, SC_P_MINV));
}

// the pressure PCG with the spectral preconditioner (pvof_spec.cu), one
// cooperative launch per solve
int p_solve_spectral(pvof_ctx *c)
{
    const Dom &d = c->dom;
    const char *why = nullptr;
    if (!spec_supported(d, &why)) return set_err(PVOF_EINVAL, why);
    const int N = d.NX - 1, M = d.NY - 1;
    if (!c->spec_mem) {
        HostMetrics hm;   // the spacings the operator uses (idx_c[1], idy_c[1] on the device)
        build_metrics(c->g, d.NX, d.NY, hm);
        const double idx2 = hm.idx_c[1 + NG] * hm.idx_c[1 + NG], idy2 = hm.idy_c[1 + NG] * hm.idy_c[1 + NG];
        c->spec_fscale = 1.0 / (idy2 * (double)N);
        c->spec_blocks = spec_pcg_blocks(c->device, N, M);
        if (c->spec_blocks <= 0) return set_err(PVOF_ECUDA, "the spectral pressure solve needs a cooperative launch");
        std::vector<double> tw, tri;
        spec_tables(N, M, idx2, idy2, tw, tri);
        const size_t parts = 3 * (size_t)c->spec_blocks;
        std::vector<double> h(tw);
        h.resize(h.size() + parts, 0.0);
        h.insert(h.end(), tri.begin(), tri.end());
        h.resize(h.size() + 3 * c->plane_elems, 0.0);   // the face coefficients and weight roots of a solve
        if (cudaMalloc(&c->spec_mem, h.size() * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&c->spec_s, sizeof(SpecScal)) != cudaSuccess)
            return set_err(PVOF_ENOMEM, "allocating the spectral preconditioner");
        // on the context's (non-blocking) stream, so the solve's launches are
        // ordered after them; a copy or memset on the legacy default stream
        // is not, and a zeroing of the barrier state landing in the middle of
        // the first solve erased arrivals (a grid barrier timeout)
        CK(cudaMemcpyAsync(c->spec_mem, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(c->spec_s, 0, sizeof(SpecScal), c->stream));
    }
    SpecArgs A;
    A.d = d;
    A.mp = c->maps[BK_PRESSURE];
    A.phi = F(c, PVOF_F_DELTAP);
    A.rhs = F(c, PVOF_F_P_RHS);
    A.rho = F(c, PVOF_F_RHO);
    A.MJ = S(c, SC_P_MINV);
    A.res = S(c, SC_P_RES);
    A.z = S(c, SC_P_Z);
    A.Ad = S(c, SC_P_AD);
    A.hat = S(c, SC_P_HAT);
    A.tw = reinterpret_cast<const double2 *>(c->spec_mem);
    A.part = c->spec_mem + N;
    A.tri = A.part + 3 * (size_t)c->spec_blocks;
    {
        const int NW = N / 2 + 1;
        const int P = M / 2 < 32 ? M / 2 : 32;   // spec_tables' chunk rule: P chunks, K the longest
        const int K = M / P + (M % P ? 1 : 0);
        double *planes = const_cast<double *>(A.tri) + (size_t)NW * (2 * K + 4) * 32;
        A.cx = planes + (size_t)OY * c->dom.P + OX;
        A.cy = A.cx + c->plane_elems;
        A.sm = A.cy + c->plane_elems;
    }
    A.N = N;
    A.R = N % 3 == 0 ? 3 : (N % 5 == 0 ? 5 : 1);
    A.n = N / A.R;
    A.logN = 0;
    while ((1 << A.logN) < A.n) A.logN++;
    A.M = M;
    A.fscale = c->spec_fscale;
    A.tol = c->p.P_CG_ETOL;
    A.maxit = c->p.P_CG_MAXIT;
    A.s = c->spec_s;
    A.scal = c->scal;
    TRY(timed_launch(c, PVOF_SOLVER_PRESSURE, 0, N * M, [&]() {
        return spec_launch_pcg(A, c->spec_blocks, S(c, SC_P_D), S(c, SC_P_D2), c->stream);
    }));
    return fill(c, BK_WRAP_C, F(c, PVOF_F_DELTAP));
}

// The grid-wide pressure solver for the context's range: the passes over
// pairs of cells (16-byte accesses) once every resident thread has at least
// two cells, single cells below that, where a pair only lengthens the
// thread's chain of loads (B200, per iteration: 2048x2048 94.0 -> 86.9 us,
// 1024x1024 20.7 -> 19.9 us with pairs; 256x512 8.2 us with single cells,
// 8.7 with pairs).
bool grid_pressure_pairs(const pvof_ctx *c)
{
    if (c->pressure_pairs >= 0) return c->pressure_pairs != 0;
    const long long n = (long long)(c->dom.NX - 1) * (c->dom.NY - 1);
    return n >= 2LL * c->coop_blocks_of[PVOF_SOLVER_PRESSURE] * COOP_THREADS;
}

const void *grid_pressure_kernel(const pvof_ctx *c)
{
    return grid_pressure_pairs(c) ? (const void *)k_cg_pressure_fwp : (const void *)k_cg_pressure_fw;
}

int p_solve(pvof_ctx *c)
{
    if (c->p.pressure_preconditioner != 0) return p_solve_spectral(c);
    PresArgs A;
    A.d = c->dom;
    A.mp = c->maps[BK_PRESSURE];
    A.phi = F(c, PVOF_F_DELTAP);
    A.rhs = F(c, PVOF_F_P_RHS);
    A.rho = F(c, PVOF_F_RHO);
    A.M = S(c, SC_P_MINV);
    A.res = S(c, SC_P_RES);
    A.dir = S(c, SC_P_D);
    A.dir2 = S(c, SC_P_D2);
    A.z = S(c, SC_P_Z);
    A.Ad = S(c, SC_P_AD);
    A.tol = c->p.P_CG_ETOL;
    A.maxit = c->p.P_CG_MAXIT;
    A.partials = c->partials;
    A.scal = c->scal;
    A.bx = S(c, SC_P_BX);
    A.by = S(c, SC_P_BY);
    const int n = (c->dom.NX - 1) * (c->dom.NY - 1);
    if (c->cgs_p_smem)
        TRY(timed_launch(c, PVOF_SOLVER_PRESSURE, 0, n, [&]() { return cgs_pressure_launch(A, StripPlan{c->cgs_p_smem, c->cgs_p_threads}, c->stream); }));
    else
        TRY(coop_launch(c, grid_pressure_kernel(c), A, n, PVOF_SOLVER_PRESSURE, 0));
    return fill(c, BK_WRAP_C, F(c, PVOF_F_DELTAP));
}

int p_project(pvof_ctx *c)
{
    double *dp = F(c, PVOF_F_DELTAP), *pd = F(c, PVOF_F_P);
    TRY(fill(c, BK_PRESSURE, dp));
    TRY(launch2d(c, k_p_update, 0, c->dom.NX - 1, 0, c->dom.NY - 1, pd, (const double *)dp));
    TRY(fill(c, BK_PRESSURE, pd));
    double mdt = 2.0 * bet(c->stage) * c->dt;
    int i0, i1, j0, j1;
    u_range(c, i0, i1, j0, j1);
    TRY(launch2d(c, k_project, i0, i1, j0, j1, 0, F(c, PVOF_F_U), (const double *)dp, (const double *)F(c, PVOF_F_RHO), mdt));
    v_range(c, i0, i1, j0, j1);
    return launch2d(c, k_project, i0, i1, j0, j1, 1, F(c, PVOF_F_V), (const double *)dp, (const double *)F(c, PVOF_F_RHO), mdt);
}

int p_divergence_async(pvof_ctx *c)
{
    CK(cudaMemsetAsync(&c->scal->div_max, 0, sizeof(double), c->stream));
    return launch2d(c, k_div_max, 0, c->dom.NX - 1, 0, c->dom.NY - 1, (const double *)F(c, PVOF_F_U),
                    (const double *)F(c, PVOF_F_V), (unsigned long long *)&c->scal->div_max);
}

int read_scalars(pvof_ctx *c)
{
    CK(cudaMemcpyAsync(c->scal_host, c->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->npend) collect_solver_timing(c);
    collect_tune(c);
    if (c->scal_host->error) {
        const int code = c->scal_host->error;
        CK(cudaMemsetAsync(c->scal, 0, sizeof(DevScalars), c->stream));
        if (c->spec_s) CK(cudaMemsetAsync(c->spec_s, 0, sizeof(SpecScal), c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return set_err(PVOF_ECUDA, code == 4 ? "advection tile load timed out"
                                   : code == 3 ? "cluster solver: a slab edge outside the owner's boundary rows"
                                              : code == 2 ? "solver grid barrier timed out (spectral pressure solve)"
                                                          : "solver grid barrier timed out (grid-wide solver)");
    }
    return PVOF_OK;
}

void fill_stats(pvof_ctx *c, pvof_stats *st)
{
    if (!st) return;
    const DevScalars &h = *c->scal_host;
    st->ch_iters = h.ch_iters;
    st->ch_rel_res = h.ch_rel;
    st->u_iters = h.vel_iters[0];
    st->v_iters = h.vel_iters[1];
    st->u_rms = h.vel_rms[0];
    st->v_rms = h.vel_rms[1];
    st->p_iters = h.p_iters;
    st->p_res = h.p_res;
    st->div_max = h.div_max;
    st->clamp_mass = h.clamp_delta;
}

int initialize(pvof_ctx *c)
{
    TRY(fill(c, BK_U, F(c, PVOF_F_U)));
    TRY(fill(c, BK_V, F(c, PVOF_F_V)));
    TRY(fill(c, BK_PRESSURE, F(c, PVOF_F_P)));
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_F)));
    TRY(vof_diffuse_init(c));
    TRY(update_density_viscosity(c));
    if (c->p.surface_tension) {
        TRY(compute_psi_LG(c));
        if (resolved(c)) TRY(extend_psi_LG(c));
        TRY(compute_f_sigma(c));
        size_t bytes = c->plane_elems * sizeof(double);
        CK(cudaMemcpyAsync(c->base[PVOF_F_FSIG_OLD_X], c->base[PVOF_F_FSIG_NEW_X], bytes, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(c->base[PVOF_F_FSIG_OLD_Y], c->base[PVOF_F_FSIG_NEW_Y], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    if (resolved(c)) TRY(ibm_velocity_init(c));   // Cart3d.c:505-515
    c->phi_prev_mask = 0;
    c->phi_old_mask = 0;
    TRY(cell_center(c));
    c->time = 0.0;
    c->clamp_total = 0.0;
    return PVOF_OK;
}

int poisson_pass(pvof_ctx *c, bool warm);

// Temporal_int_all_the_equations (Temporal_int.c:563-1279) up to the first
// Poisson pass's divergence check; with resolved particles the branches of
// VOF_IBM and LAG_PARTICLE_RESOLVED
int substep_region(pvof_ctx *c, bool warm0)
{
    const bool solids = resolved(c);
    if (c->stage > 0) TRY(cell_center(c));
    TRY(fill(c, BK_WRAP_C, F(c, PVOF_F_U_BC)));
    TRY(fill(c, BK_WRAP_C, F(c, PVOF_F_V_BC)));
    if (solids) {
        TRY(ibm_flag_points(c));   // Particle_MPI_update of both lists, Lagrangian_flag_points
        TRY(compute_C_S(c));
    }
    TRY(vof_diffuse_step(c));
    TRY(update_density_viscosity(c));
    TRY(implicit_explicit(c, 0));
    TRY(implicit_explicit(c, 1));
    TRY(set_rhs(c, 0));
    TRY(set_rhs(c, 1));
    if (c->p.surface_tension) {
        TRY(compute_psi_LG(c));
        if (solids && c->stage == 2) TRY(extend_psi_LG(c));
        TRY(compute_f_sigma(c));
        TRY(apply_f_sigma_old(c));
    }
    if (c->p.gravity) TRY(add_gravity(c));
    if (solids) {
        // explicit predictor and direct forcing on the right-hand side (Temporal_int.c:948-980)
        TRY(vel_explicit(c, 0));
        TRY(vel_explicit(c, 1));
        TRY(fill(c, BK_U, F(c, PVOF_F_U)));
        TRY(fill(c, BK_V, F(c, PVOF_F_V)));
        TRY(ibm_force(c, -1));
    }
    TRY(velocity_solve_both(c));
    TRY(fill(c, BK_U, F(c, PVOF_F_U)));
    TRY(fill(c, BK_V, F(c, PVOF_F_V)));
    if (solids) {
        // forcing correctors on the velocity (Temporal_int.c:1008-1022)
        TRY(ibm_force(c, c->p.N_forcing_loops));
        TRY(fill(c, BK_U, F(c, PVOF_F_U)));
        TRY(fill(c, BK_V, F(c, PVOF_F_V)));
    }
    return poisson_pass(c, warm0);
}

// one pass of the outer Poisson loop up to its divergence check (read by the host)
int poisson_pass(pvof_ctx *c, bool warm)
{
    TRY(p_set_rhs(c, warm));
    TRY(p_precond(c));
    TRY(p_solve(c));
    TRY(p_project(c));
    TRY(fill(c, BK_U, F(c, PVOF_F_U)));
    TRY(fill(c, BK_V, F(c, PVOF_F_V)));
    return p_divergence_async(c);
}

// The region above as a CUDA graph.  Its launches and their arguments depend
// on the host state in GraphKey only (resolved particles included: their
// bookkeeping runs on the device, its launches cover the capacities set by
// pvof_set_particles, which drops the captured graphs; without the learned
// warm start, and without solver timing, whose events must be recorded
// launch by launch); a key is
// captured the second time it is seen, so lazy set-up (allocations, tables)
// has run outside the capture, and replayed after that.  A key whose capture
// fails runs its launches directly from then on.
bool graph_key_equal(const GraphKey &a, const GraphKey &b)
{
    return a.stage == b.stage && a.dt == b.dt && a.fsig == b.fsig && a.warm == b.warm &&
           a.one_cluster == b.one_cluster;
}

// The solver kernels whose blocks wait on one another (grid barriers) must
// stay cooperative launches, all blocks co-resident, when replayed from a
// graph: mark their kernel nodes so explicitly.  False if a node could not be
// read or marked.
bool keep_cooperative(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return false;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return false;
    const void *coop[] = {(const void *)k_cg_biharmonic, (const void *)k_cg_velocity, (const void *)k_cg_pressure_fw,
                          (const void *)k_cg_pressure_fwp,
                          spec_pcg_kernel()};
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) return false;
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess) return false;
        for (const void *f : coop) {
            if (kp.func != f) continue;
            cudaLaunchAttributeValue v;
            std::memset(&v, 0, sizeof(v));
            v.cooperative = 1;
            if (cudaGraphKernelNodeSetAttribute(nd, cudaLaunchAttributeCooperative, &v) != cudaSuccess) return false;
        }
    }
    return true;
}

// waits for the context's stream and drops its captured substeps (after a
// change of the launches or buffers they hold)
void drop_graphs(pvof_ctx *c)
{
    cudaStreamSynchronize(c->stream);
    for (GraphEntry &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = GraphEntry();
    }
    c->graph_next = 0;
}

int run_region(pvof_ctx *c, bool warm0)
{
    if (!c->use_graphs || c->solver_timing || (c->tune && c->tune->active) || c->p.pressure_warm_start == 2)
        return substep_region(c, warm0);
    GraphKey k;
    k.stage = c->stage;
    k.dt = c->dt;
    k.fsig = c->f[PVOF_F_FSIG_OLD_X];
    k.warm = warm0 ? 1 : 0;
    k.one_cluster = c->vel_one_cluster;
    GraphEntry *e = nullptr;
    for (GraphEntry &g : c->graphs)
        if (g.state != 0 && graph_key_equal(g.key, k)) { e = &g; break; }
    if (!e) {   // first sight: remember the key, run directly
        GraphEntry &g = c->graphs[c->graph_next];
        c->graph_next = (c->graph_next + 1) % Ctx::NGRAPHS;
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = GraphEntry();
        g.key = k;
        g.state = 1;
        return substep_region(c, warm0);
    }
    if (e->state == 3) return substep_region(c, warm0);
    if (e->state == 1) {   // second sight: capture
        const long long l0 = c->launches;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            e->state = 3;
            return substep_region(c, warm0);
        }
        const int rc = substep_region(c, warm0);
        cudaGraph_t g = nullptr;
        cudaError_t ee = cudaStreamEndCapture(c->stream, &g);
        cudaGraphExec_t x = nullptr;
        if (rc == PVOF_OK && ee == cudaSuccess && g && !keep_cooperative(g)) ee = cudaErrorUnknown;
        if (rc == PVOF_OK && ee == cudaSuccess && g) ee = cudaGraphInstantiate(&x, g, 0);
        if (g) cudaGraphDestroy(g);
        if (rc != PVOF_OK || ee != cudaSuccess || !x) {
            if (x) cudaGraphExecDestroy(x);
            cudaGetLastError();
            e->state = 3;
            c->launches = l0;
            return substep_region(c, warm0);
        }
        e->exec = x;
        e->state = 2;
        e->launches = c->launches - l0;
        c->launches = l0;
    }
    CK(cudaGraphLaunch(e->exec, c->stream));
    c->graph_replays++;
    c->launches += e->launches;
    return PVOF_OK;
}

// Temporal_int_all_the_equations (Temporal_int.c:563-1279); with resolved
// particles the branches of VOF_IBM and LAG_PARTICLE_RESOLVED
int substep(pvof_ctx *c, pvof_stats *st)
{
    const bool solids = resolved(c);
    const bool warm0 = c->p.pressure_warm_start && (c->phi_prev_mask >> c->stage & 1);
    TRY(run_region(c, warm0));
    int passes = 0, p_total = 0;
    int rc = PVOF_OK;
    for (;;) {
        if (passes > 0) TRY(poisson_pass(c, false));
        TRY(read_scalars(c));
        passes++;
        p_total += c->scal_host->p_iters;
        if (passes > 10) { rc = set_err(PVOF_EDIVERGED, "Poisson solver did not converge"); break; }
        if (!(c->scal_host->div_max > 1e-6)) break;
    }
    if (c->p.pressure_warm_start && rc == PVOF_OK) {
        const size_t bytes = c->plane_elems * sizeof(double);
        if (c->phi_prev_mask >> c->stage & 1) {   // one generation back, for the network's samples
            CK(cudaMemcpyAsync(c->sbase[SC_PHI_OLD + c->stage], c->sbase[SC_PHI_PREV + c->stage], bytes,
                               cudaMemcpyDeviceToDevice, c->stream));
            c->phi_old_mask |= 1 << c->stage;
        }
        CK(cudaMemcpyAsync(c->sbase[SC_PHI_PREV + c->stage], c->base[PVOF_F_DELTAP], bytes, cudaMemcpyDeviceToDevice,
                           c->stream));
        c->phi_prev_mask |= 1 << c->stage;
    }
    c->clamp_total += c->scal_host->clamp_delta;
    if (c->p.surface_tension) swap_f_sigma(c);
    if (solids && rc == PVOF_OK) TRY(ibm_advect(c));   // Temporal_int.c:1186-1238
    if (st) {
        fill_stats(c, st);
        st->p_iters_total = p_total;
        st->poisson_passes = passes;
    }
    return rc;
}

// ---------------------------------------------------------------------------
// resolved solid particles (kernels and list bookkeeping in pvof_ibm.cu)
// ---------------------------------------------------------------------------
}  // namespace

struct pvof::IbmState {
    HostMetrics hm;
    PSet P;                                // host copy: pointers, capacities, grid; counts as last set by the host
    PSet *d_ps = nullptr;                  // the device copy the kernels update
    double *d_coord = nullptr;             // xu, xc, yv, yc, each offset by NG
    const double *xu = nullptr, *xc = nullptr, *yv = nullptr, *yc = nullptr;
    char *d_mem = nullptr;                 // every buffer of P, one allocation
    bool flagged = false;
    ~IbmState()
    {
        cudaFree(d_mem);
        cudaFree(d_ps);
        cudaFree(d_coord);
    }
};

namespace {

int ibm_state(pvof_ctx *c, IbmState **out)
{
    if (c->ibm) { *out = c->ibm; return PVOF_OK; }
    IbmState *s = new IbmState();
    std::memset(&s->P, 0, sizeof(PSet));
    build_metrics(c->g, c->dom.NX, c->dom.NY, s->hm);
    const size_t nx = s->hm.xu.size(), ny = s->hm.yv.size();
    if (cudaMalloc(&s->d_coord, (2 * nx + 2 * ny) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s->d_ps, sizeof(PSet)) != cudaSuccess) {
        delete s;
        return set_err(PVOF_ENOMEM, "cudaMalloc particle state");
    }
    std::vector<double> h;
    for (auto *v : {&s->hm.xu, &s->hm.xc, &s->hm.yv, &s->hm.yc}) h.insert(h.end(), v->begin(), v->end());
    CK(cudaMemcpyAsync(s->d_coord, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    s->xu = s->d_coord + NG;
    s->xc = s->d_coord + nx + NG;
    s->yv = s->d_coord + 2 * nx + NG;
    s->yc = s->d_coord + 2 * nx + ny + NG;
    PGrid &g = s->P.g;
    const int NX = c->dom.NX, NY = c->dom.NY;
    g.NX = NX;
    g.NY = NY;
    g.periodic[0] = c->dom.perx;
    g.periodic[1] = c->dom.pery;
    g.axisym = c->dom.axisym;
    g.h = s->hm.dx_u[1 + NG];
    double dymin = s->hm.dy_v[NG];
    for (int j = 0; j < NY; j++) dymin = std::min(dymin, s->hm.dy_v[j + NG]);
    g.dy_min = dymin;
    g.slab = c->dom.slab;
    g.twod_slab = c->g.slab_thickness;
    g.Lx = c->g.xmax - c->g.xmin;
    g.Ly = c->g.ymax - c->g.ymin;
    g.zs = c->g.zmin + 0.5 * (c->g.zmax - c->g.zmin);   // zc[G_Ks] of the storage plane
    g.xu0 = s->hm.xu[NG];
    g.xuN = s->hm.xu[NX - 1 + NG];
    g.yv0 = s->hm.yv[NG];
    g.yvN = s->hm.yv[NY - 1 + NG];
    g.xcm1 = s->hm.xc[NG - 1];
    g.ycm1 = s->hm.yc[NG - 1];
    c->ibm = s;
    *out = s;
    return PVOF_OK;
}

// the particle state of a context in the resolved-particle mode
int ibm_need(pvof_ctx *c, IbmState **out)
{
    if (!c->ibm || !c->ibm->d_mem) return set_err(PVOF_EINVAL, "pvof_set_particles() first");
    *out = c->ibm;
    return PVOF_OK;
}

// the device copy's counts and error state (waits for the stream)
int ibm_read(pvof_ctx *c, IbmState *s, PSet &h)
{
    CK(cudaMemcpyAsync(&h, s->d_ps, sizeof(PSet), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PVOF_OK;
}

// the bookkeeping's error state as an error code and message
int ibm_check(pvof_ctx *c, IbmState *s)
{
    PSet h;
    TRY(ibm_read(c, s, h));
    if (h.err == 0) return PVOF_OK;
    char msg[256];
    if (h.err == 1 && h.err_b >= 0)
        snprintf(msg, sizeof(msg), "particles %d and %d within the lubrication range: the collision models are not built",
                 h.err_a, h.err_b);
    else if (h.err == 1)
        snprintf(msg, sizeof(msg), "particle %d within the lubrication range of a wall: the collision models are not built",
                 h.err_a);
    else
        snprintf(msg, sizeof(msg), "the particle lists or markers outgrew their capacity");
    return set_err(PVOF_EINVAL, msg);
}

// Particle_MPI_update of both lists and Lagrangian_flag_points
// (Temporal_int.c:678-681), on the device
int ibm_flag_points(pvof_ctx *c)
{
    IbmState *s;
    TRY(ibm_need(c, &s));
    k_ps_update<<<1, 32, 0, c->stream>>>(s->d_ps);
    CKL(c);
    k_ps_markers<<<1, PS_MARKER_THREADS, 0, c->stream>>>(s->d_ps);
    CKL(c);
    s->flagged = true;
    return PVOF_OK;
}

IbmDev ibm_dev(pvof_ctx *c, IbmState *s)
{
    const PSet &P = s->P;
    const size_t cap = (size_t)P.cap_mk;
    IbmDev D;
    D.ent = P.dent;
    D.ne = &s->d_ps->ne;
    D.XL = P.mk;
    D.YL = P.mk + cap;
    D.vol = P.mk + 2 * cap;
    D.UL = P.mk + 3 * cap;
    D.rhoL = P.mk + 4 * cap;
    D.FL = P.mk + 5 * cap;
    D.flag = P.mflag;
    D.sup_i = P.mflag + cap;
    D.sup_j = P.mflag + 2 * cap;
    D.FT = P.FT;
    D.xlo = P.g.xu0;
    D.xhi = P.g.xuN;
    D.ylo = P.g.yv0;
    D.yhi = P.g.yvN;
    D.h = P.g.h;
    D.dxu1 = s->hm.dx_u[1 + NG];
    D.slab = c->dom.slab > 0.0 ? c->dom.slab : D.dxu1;
    D.dyv = c->dom.m.dy_v;
    D.axisym = c->dom.axisym;
    D.theta_span = c->g.theta_span;
    return D;
}

// Lagrangian_force (Lagrangian.c:1724-1871) without the squirmer, one-way and
// post-processing options.  The marker and entry launches cover the
// capacities and read the counts on the device.
int ibm_force(pvof_ctx *c, int force_iter)
{
    IbmState *s = c->ibm;
    if (!s || !s->flagged) return set_err(PVOF_EINVAL, "pvof_Lagrangian_flag_points() first");
    const Dom &d = c->dom;
    const int NX = d.NX, NY = d.NY;
    const double dtbeta = bet(c->stage) * c->dt;
    const double idt2beta = 1.0 / (2.0 * bet(c->stage) * c->dt);
    const int corrector = force_iter >= 0, iters = corrector ? force_iter : 1;
    IbmDev D = ibm_dev(c, s);
    const int *nm = &s->d_ps->nm;
    const dim3 cb(128), cg((unsigned)((NX + 127) / 128), (unsigned)NY);
    const unsigned mg = (unsigned)((s->P.cap_mk + 127) / 128), eg = (unsigned)s->P.cap_ent;
    double *U = F(c, PVOF_F_U), *V = F(c, PVOF_F_V), *RU = F(c, PVOF_F_U_RHS), *RV = F(c, PVOF_F_V_RHS);
    const double *rho = F(c, PVOF_F_RHO);
    for (int ii = 0; ii < iters; ii++) {
        TRY(fill(c, BK_WRAP_U, U));
        TRY(fill(c, BK_WRAP_V, V));
        if (corrector) {
            k_ibm_ng_update<<<cg, cb, 0, c->stream>>>(d, RU, nullptr, 1);
            CKL(c);
            k_ibm_ng_update<<<cg, cb, 0, c->stream>>>(d, RV, nullptr, 1);
            CKL(c);
        }
        k_ibm_interp<<<mg, 128, 0, c->stream>>>(d, rho, s->xc, s->yc, D.h, D.XL, D.YL, nm,
                                                d.axisym ? IBM_AXIS_EVEN : IBM_AXIS_NONE, D.rhoL);
        CKL(c);
        for (int comp = 0; comp < 2; comp++) {
            const double *xs = comp == 0 ? s->xu : s->xc, *ys = comp == 0 ? s->yc : s->yv;
            const int axis = !d.axisym ? IBM_AXIS_NONE : (comp == 0 ? IBM_AXIS_ODD : IBM_AXIS_EVEN);
            k_ibm_interp<<<mg, 128, 0, c->stream>>>(d, comp == 0 ? U : V, xs, ys, D.h, D.XL, D.YL, nm, axis, D.UL);
            CKL(c);
            const double xs0 = comp == 0 ? s->hm.xu[NG] : s->hm.xc[NG];
            const double ys0 = comp == 0 ? s->hm.yc[NG] : s->hm.yv[NG];
            k_ibm_marker_force<<<eg, IBM_FORCE_THREADS, 0, c->stream>>>(D, comp, xs0, ys0, idt2beta,
                                                                        (!corrector && comp == 0) ? 1 : 0);
            CKL(c);
            k_ibm_spread<<<cg, cb, 0, c->stream>>>(d, D, comp, xs, ys, rho, comp == 0 ? RU : RV);
            CKL(c);
        }
        if (corrector) {
            k_ibm_correct<<<cg, cb, 0, c->stream>>>(d, 0, dtbeta, RU, rho, U);
            CKL(c);
            k_ibm_correct<<<cg, cb, 0, c->stream>>>(d, 1, dtbeta, RV, rho, V);
            CKL(c);
        }
    }
    if (!corrector) {
        k_ibm_ng_update<<<cg, cb, 0, c->stream>>>(d, RU, F(c, PVOF_F_U_IMPLICIT), 0);
        CKL(c);
        k_ibm_ng_update<<<cg, cb, 0, c->stream>>>(d, RV, F(c, PVOF_F_V_IMPLICIT), 0);
        CKL(c);
    }
    return PVOF_OK;
}

// Velocity_solve_explicit (msolve_direct.c:146-260)
int vel_explicit(pvof_ctx *c, int comp)
{
    int i0, i1, j0, j1;
    if (comp == 0) u_range(c, i0, i1, j0, j1);
    else v_range(c, i0, i1, j0, j1);
    if (i1 <= i0 || j1 <= j0) return PVOF_OK;
    const dim3 cb(128), cg((unsigned)((i1 - i0 + 127) / 128), (unsigned)(j1 - j0));
    k_vel_explicit<<<cg, cb, 0, c->stream>>>(c->dom, comp, i0, i1, j0, j1, bet(c->stage) * c->dt,
                                              F(c, comp == 0 ? PVOF_F_U_RHS : PVOF_F_V_RHS), F(c, PVOF_F_RHO),
                                              F(c, comp == 0 ? PVOF_F_U : PVOF_F_V));
    CKL(c);
    return PVOF_OK;
}

// VOF_DIFFUSE_compute_C_S (VOF_DIFFUSE.c:685-813): the particles' geometry
// from the owned lists on the device, then the field
int compute_C_S(pvof_ctx *c)
{
    IbmState *s;
    TRY(ibm_need(c, &s));
    k_ps_geo<<<1, 32, 0, c->stream>>>(s->d_ps);
    CKL(c);
    double shift, denom, extra;
    ibm_solid_constants(c->p.Cn, shift, denom, extra);
    const Dom &d = c->dom;
    const dim3 cb(128), cg((unsigned)((d.NX + 2 * NG + 127) / 128), (unsigned)(d.NY + 2 * NG));
    k_compute_C_S<<<cg, cb, 0, c->stream>>>(d, s->xc, s->yc, s->P.geo, &s->d_ps->ngeo, shift, denom, extra,
                                             F(c, PVOF_F_C_S));
    CKL(c);
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_C_S)));
    TRY(bound(c));
    TRY(fill(c, BK_SCALAR, F(c, PVOF_F_C_L)));
    TRY(phase_cache(c));
    return fill(c, BK_SCALAR, F(c, PVOF_F_C_G));
}

// per-entry momentum integrals (and with ccf the capillary contact force) of
// the current list entries, into the device's sums
int ibm_sums(pvof_ctx *c, bool ccf)
{
    IbmState *s = c->ibm;
    IbmSumArgs A;
    A.ent = s->P.dent;
    A.ne = &s->d_ps->ne;
    A.U = F(c, PVOF_F_U);
    A.V = F(c, PVOF_F_V);
    A.CL = F(c, PVOF_F_C_L);
    A.CS = F(c, PVOF_F_C_S);
    A.xu = s->xu;
    A.xc = s->xc;
    A.yv = s->yv;
    A.yc = s->yc;
    A.plist = s->P.plist;
    A.np = &s->d_ps->np;
    A.h = s->P.g.h;
    A.slab = c->dom.slab > 0.0 ? c->dom.slab : s->P.g.h;   // Interpolate_twod_cell_volume
    A.sigma = 1.0 / c->p.We;
    const double theta = c->p.contact_angle_deg * M_PI / 180.0;
    A.ct = std::cos(theta);
    A.st = std::sin(theta);
    const double epsN = 1.0e-14;
    const double h_ref = (s->P.g.dy_min > epsN) ? s->P.g.dy_min : epsN;
    const double cn = (c->p.Cn > 0.0) ? c->p.Cn : 0.0;
    A.support_width = 8.0 * ((cn > h_ref) ? cn : h_ref);
    A.nk = c->dom.nk;
    A.ccf = ccf ? 1 : 0;
    A.axisym = c->dom.axisym;
    A.theta_span = c->g.theta_span;
    A.out = s->P.sums;
    k_ibm_particle_sums<<<(unsigned)s->P.cap_ent, 256, 0, c->stream>>>(c->dom, A);
    CKL(c);
    return PVOF_OK;
}

// the end of a substep with resolved particles (Temporal_int.c:1186-1238):
// momentum integrals and contact-line forces of every list entry, their
// collection into the owned particles and Lagrangian_advect_particles, all on
// the device; the host reads back only the error state
int ibm_advect(pvof_ctx *c)
{
    IbmState *s = c->ibm;
    if (!s || !s->flagged) return set_err(PVOF_EINVAL, "pvof_Lagrangian_flag_points() first");
    TRY(ibm_sums(c, true));
    k_ps_collect<<<1, 32, 0, c->stream>>>(s->d_ps, PS_ADVANCE, 1, c->stage, c->dt);
    CKL(c);
    return ibm_check(c, s);
}

// Particle_initialize_velocities (Lagrangian/Particle.c:322-535): mobile
// particles take the volume-averaged fluid velocity, the fluid inside them is
// painted to that rigid motion, and the momentum integrals of the painted
// field become the reference for the first rigid-body force
int ibm_velocity_init(pvof_ctx *c)
{
    IbmState *s = c->ibm;
    TRY(ibm_flag_points(c));
    TRY(ibm_sums(c, false));
    k_ps_collect<<<1, 32, 0, c->stream>>>(s->d_ps, PS_INIT_VELOCITY, 0, 0, 0.0);
    CKL(c);
    TRY(ibm_flag_points(c));
    double *U = F(c, PVOF_F_U), *V = F(c, PVOF_F_V);
    const dim3 blk(16, 16), grd((unsigned)((c->dom.NX + 15) / 16), (unsigned)((c->dom.NY + 15) / 16));
    for (int comp = 0; comp < 2; comp++) {
        k_ps_paint<<<grd, blk, 0, c->stream>>>(c->dom, s->d_ps, comp, s->xu, s->xc, s->yv, s->yc, comp == 0 ? U : V);
        CKL(c);
    }
    TRY(fill(c, BK_WRAP_U, U));
    TRY(fill(c, BK_WRAP_V, V));
    TRY(fill(c, BK_U, U));
    TRY(fill(c, BK_V, V));
    TRY(ibm_sums(c, false));
    k_ps_collect<<<1, 32, 0, c->stream>>>(s->d_ps, PS_INIT_MOMENTUM, 0, 0, 0.0);
    CKL(c);
    return ibm_check(c, s);
}

// contact-line projection (VOF_IBM_wetting.c:1021-2131; kernels in pvof_mcl.cu)
int mcl_normals(pvof_ctx *c)
{
    IbmState *s;
    TRY(ibm_need(c, &s));
    const Dom &d = c->dom;
    const double h_ref = (s->P.g.dy_min > 0.0) ? s->P.g.dy_min : 1.0e-14;
    const double cn = (c->p.Cn > 0.0) ? c->p.Cn : 0.0;
    const double support_width = 8.0 * ((cn > h_ref) ? cn : h_ref);
    const dim3 blk(128), grd((unsigned)((d.NX + 2 * NG + 127) / 128), (unsigned)(d.NY + 2 * NG));
    k_mcl_normals<<<grd, blk, 0, c->stream>>>(d, s->xc, s->yc, F(c, PVOF_F_C_S), s->P.plist, &s->d_ps->np,
                                              support_width, F(c, PVOF_F_NX_IBM), F(c, PVOF_F_NY_IBM));
    CKL(c);
    if (d.axisym) {
        k_mcl_axis_normals<<<(unsigned)((d.NY + 2 * NG + 127) / 128), 128, 0, c->stream>>>(d, F(c, PVOF_F_NX_IBM),
                                                                                         F(c, PVOF_F_NY_IBM));
        CKL(c);
    }
    TRY(fill(c, BK_NRM_X, F(c, PVOF_F_NX_IBM)));
    return fill(c, BK_NRM_Y, F(c, PVOF_F_NY_IBM));
}

MclView mcl_view(pvof_ctx *c, const double *CL, const double *field)
{
    IbmState *s = c->ibm;
    MclView v;
    v.NX = c->dom.NX;
    v.NY = c->dom.NY;
    v.perx = c->dom.perx;
    v.pery = c->dom.pery;
    v.free_lo_x = !v.perx && c->g.wall[PVOF_LEFT] == PVOF_WALL_FREESLIP;
    v.free_hi_x = !v.perx && c->g.wall[PVOF_RIGHT] == PVOF_WALL_FREESLIP;
    v.free_lo_y = !v.pery && c->g.wall[PVOF_BOTTOM] == PVOF_WALL_FREESLIP;
    v.free_hi_y = !v.pery && c->g.wall[PVOF_TOP] == PVOF_WALL_FREESLIP;
    v.xc = s->xc;
    v.yc = s->yc;
    // theta and its cosine and sine as the reference forms them (:1987-1988)
    const double theta = c->p.contact_angle_deg * M_PI / 180.0;
    v.ct = std::cos(theta);
    v.st = std::sin(theta);
    v.hydrophilic = theta <= 0.5 * M_PI;
    // mcl_lg_band_limits (:862-877)
    v.cmin = 0.005;
    v.cmax = 0.995;
    if (c->p.contact_angle_deg > 0.0 && c->p.contact_angle_deg < 45.0) {
        v.cmin = 0.05;
        v.cmax = 0.95;
    }
    v.CS = F(c, PVOF_F_C_S);
    v.CG = F(c, PVOF_F_C_G);
    v.CL = CL;
    v.field = field;
    return v;
}

// VOF_DIFFUSE_apply_contact_angle (:1946-2008): one pass over a snapshot of C_L
int apply_contact_angle(pvof_ctx *c)
{
    TRY(mcl_normals(c));
    double *CL = F(c, PVOF_F_C_L), *snap = S(c, SC_SNAP);
    CK(cudaMemcpyAsync(c->sbase[SC_SNAP], c->base[PVOF_F_C_L], c->plane_elems * sizeof(double),
                       cudaMemcpyDeviceToDevice, c->stream));
    const MclView v = mcl_view(c, snap, snap);
    const dim3 blk(128), grd((unsigned)((c->dom.NX + 127) / 128), (unsigned)c->dom.NY);
    k_mcl_apply<<<grd, blk, 0, c->stream>>>(c->dom, v, F(c, PVOF_F_NX_IBM), F(c, PVOF_F_NY_IBM), CL);
    CKL(c);
    return PVOF_OK;
}

// VOF_DIFFUSE_extend_psi_LG_contact_angle (:2014-2131)
int extend_psi_LG(pvof_ctx *c)
{
    TRY(mcl_normals(c));
    double *psi = F(c, PVOF_F_PSI_LG), *snap = S(c, SC_SNAP);
    CK(cudaMemcpyAsync(c->sbase[SC_SNAP], c->base[PVOF_F_PSI_LG], c->plane_elems * sizeof(double),
                       cudaMemcpyDeviceToDevice, c->stream));
    const MclView v = mcl_view(c, F(c, PVOF_F_C_L), snap);
    const dim3 blk(128), grd((unsigned)((c->dom.NX + 127) / 128), (unsigned)c->dom.NY);
    k_mcl_extend_psi<<<grd, blk, 0, c->stream>>>(c->dom, v, F(c, PVOF_F_NX_IBM), F(c, PVOF_F_NY_IBM), psi);
    CKL(c);
    return fill(c, BK_SCALAR, psi);
}

int p_solve_fft(pvof_ctx *c)
{
    const Dom &d = c->dom;
    if (!d.planar || !d.perx || d.pery)
        return set_err(PVOF_EINVAL, "the FFT Poisson solver needs the planar mode, x periodic and walls in y");
    const int N = d.NX - 1, NYp = d.NY - 1;
    if (N > 2048) return set_err(PVOF_EINVAL, "the FFT Poisson solver takes at most 2048 cells in x");
    int logN = -1;
    if ((N & (N - 1)) == 0) { logN = 0; while ((1 << logN) < N) logN++; }
    if (!c->fft_coef) {
        // Pressure_calc_coeff (psolve_fft.c:467-591), walls in y, x periodic
        HostMetrics hm;
        build_metrics(c->g, d.NX, d.NY, hm);
        auto idy_v = [&](int j) { return hm.idy_v[j + NG]; };
        auto idy_c = [&](int j) { return hm.idy_c[j + NG]; };
        std::vector<double> co(3 * (size_t)NYp + (size_t)N, 0.0);
        double *as_ = co.data(), *ap_ = as_ + NYp, *an_ = ap_ + NYp, *mw = an_ + NYp;
        as_[0] = 0.0;
        an_[NYp - 1] = 0.0;
        for (int j = 0; j < NYp; j++) {
            if (j > 0) as_[j] = idy_v(j) * idy_c(j - 1);
            if (j < NYp - 1) an_[j] = idy_v(j) * idy_c(j);
            ap_[j] = -as_[j] - an_[j];
        }
        an_[NYp - 1] = 0.0;
        const double idx = hm.idx_u[NG];
        const double pi = 3.14159265358979323846;
        for (int i = 0; i < N; i++) {
            const int wave = i < N / 2 ? i : N - i;   // Pressure_fft_setup wave ordering
            mw[i] = 2.0 * (1 - cos(2. * pi * wave / N)) * (idx * idx);
        }
        if (cudaMalloc(&c->fft_coef, co.size() * sizeof(double)) != cudaSuccess) {
            c->fft_coef = nullptr;
            return set_err(PVOF_ENOMEM, "cudaMalloc FFT coefficients");
        }
        CK(cudaMemcpyAsync(c->fft_coef, co.data(), co.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    const double *as_ = c->fft_coef, *ap_ = as_ + NYp, *an_ = ap_ + NYp, *mw = an_ + NYp;
    double *hc = S(c, SC_P_RES), *gam = S(c, SC_P_D);
    const size_t smem = (size_t)N * sizeof(double2);
    const double inx = 1.0 / (d.NX - 1.0);
    k_fft_forward<<<(unsigned)NYp, 256, smem, c->stream>>>(d, N, logN, F(c, PVOF_F_P_RHS), hc, inx);
    CKL(c);
    k_fft_tridiag<<<(unsigned)((N + 127) / 128), 128, 0, c->stream>>>(d, N, NYp, as_, ap_, an_, mw, hc, gam);
    CKL(c);
    k_fft_inverse<<<(unsigned)NYp, 256, smem, c->stream>>>(d, N, logN, hc, F(c, PVOF_F_DELTAP));
    CKL(c);
    return PVOF_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int pvof_abi_version(void) { return PVOF_ABI_VERSION; }

const char *pvof_last_error(void) { return g_err.c_str(); }

int pvof_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int pvof_create(const pvof_grid_desc *grid, const pvof_params *params, int device, pvof_ctx **out)
{
    if (!grid || !params || !out) return set_err(PVOF_EINVAL, "null argument");
    *out = nullptr;
    if (grid->ghost_nodes != NG) return set_err(PVOF_EINVAL, "ghost_nodes must be 3");
    if (grid->geometry == PVOF_GEOM_3D) {
        if (params->Re <= 0 || params->Pe_CH <= 0 || params->Cn <= 0) return set_err(PVOF_EINVAL, "Re, Pe_CH and Cn must be positive");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(PVOF_ENODEV, "no CUDA device");
        if (device < 0 || device >= ndev) return set_err(PVOF_EINVAL, "bad device index");
        pvof3::Handle *h = nullptr;
        int rc = from3(pvof3::create(grid, params, device, &h));
        if (rc < 0) return rc;
        pvof_ctx *c = new pvof_ctx();
        std::memset(static_cast<Ctx *>(c), 0, sizeof(Ctx));
        c->g = *grid;
        c->p = *params;
        c->device = device;
        c->h3 = h;
        *out = c;
        return PVOF_OK;
    }
    if (grid->geometry != PVOF_GEOM_PLANAR && grid->geometry != PVOF_GEOM_AXISYM)
        return set_err(PVOF_EINVAL, "geometry must be PVOF_GEOM_3D, PVOF_GEOM_PLANAR or PVOF_GEOM_AXISYM");
    if (grid->NZM != 1) return set_err(PVOF_EINVAL, "2D modes need NZM == 1");
    if (grid->NXM < 8 || grid->NYM < 8) return set_err(PVOF_EINVAL, "at least 8 cells per direction");
    if (grid->geometry == PVOF_GEOM_AXISYM && grid->periodic[0]) return set_err(PVOF_EINVAL, "the axis cannot be periodic");
    if (params->Re <= 0 || params->Pe_CH <= 0 || params->Cn <= 0) return set_err(PVOF_EINVAL, "Re, Pe_CH and Cn must be positive");
    if (params->N_forcing_loops < 0) return set_err(PVOF_EINVAL, "N_forcing_loops must not be negative");
    if (params->velocity_cg_unregularized < 0 || params->velocity_cg_unregularized > 1)
        return set_err(PVOF_EINVAL, "velocity_cg_unregularized must be 0 or 1");
    if (params->pressure_preconditioner < 0 || params->pressure_preconditioner > 1)
        return set_err(PVOF_EINVAL, "pressure_preconditioner must be 0 (Jacobi) or 1 (spectral)");
    if (params->pressure_preconditioner != 0) {
        const int N = grid->NXM, M = grid->NYM;
        if (grid->geometry != PVOF_GEOM_PLANAR || !grid->periodic[0] || grid->periodic[1])
            return set_err(PVOF_EINVAL, "the spectral pressure preconditioner needs a planar grid, x periodic, walls in y");
        int odd = N;
        while (odd % 2 == 0 && odd > 1) odd /= 2;
        if (N < 2 || N % 2 != 0 || (odd != 1 && odd != 3 && odd != 5) || N > 1024 || M < 2 || M > 1024)
            return set_err(PVOF_EINVAL, "the spectral pressure preconditioner needs an x cell count of 2^a, 3 2^a or "
                                        "5 2^a up to 1024 and 2 to 1024 y cells");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(PVOF_ENODEV, "no CUDA device");
    if (device < 0 || device >= ndev) return set_err(PVOF_EINVAL, "bad device index");
    CK(cudaSetDevice(device));

    pvof_ctx *c = new pvof_ctx();
    std::memset(static_cast<Ctx *>(c), 0, sizeof(Ctx));
    c->use_graphs = 1;
    c->pressure_pairs = -1;
    c->g = *grid;
    c->p = *params;
    c->device = device;
    Dom &d = c->dom;
    d.NX = grid->NXM + 1;
    d.NY = grid->NYM + 1;
    d.P = ((d.NX + OX + NG + 1) + 31) / 32 * 32;
    d.planar = grid->geometry == PVOF_GEOM_PLANAR;
    d.axisym = grid->geometry == PVOF_GEOM_AXISYM;
    d.perx = grid->periodic[0] != 0;
    d.pery = grid->periodic[1] != 0;
    d.nk = grid->NZM + 1;
    d.slab = grid->slab_thickness;
    d.wz = d.planar ? d.slab : 1.0;
    c->plane_elems = (size_t)d.P * (size_t)(d.NY + 2 * NG);
    const size_t origin = (size_t)OY * d.P + OX;
    auto fail = [&](int code, const std::string &m) {
        pvof_destroy(c);
        return set_err(code, m);
    };
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (int q = 0; q < PVOF_F_COUNT; q++) {
        if (cudaMalloc(&c->base[q], c->plane_elems * sizeof(double)) != cudaSuccess) return fail(PVOF_ENOMEM, "cudaMalloc field");
        cudaMemset(c->base[q], 0, c->plane_elems * sizeof(double));
        c->f[q] = c->base[q] + origin;
    }
    for (int q = 0; q < SC_COUNT; q++) {
        if (cudaMalloc(&c->sbase[q], c->plane_elems * sizeof(double)) != cudaSuccess) return fail(PVOF_ENOMEM, "cudaMalloc scratch");
        cudaMemset(c->sbase[q], 0, c->plane_elems * sizeof(double));
        c->s[q] = c->sbase[q] + origin;
    }
    // metrics
    HostMetrics hm;
    build_metrics(*grid, d.NX, d.NY, hm);
    std::vector<const std::vector<double> *> mv = {&hm.idx_u, &hm.idx_c, &hm.dx_c, &hm.dx_u, &hm.r_u, &hm.r_c,
                                                   &hm.inv_r_u, &hm.inv_r_c, &hm.ring_wt_c,
                                                   &hm.idy_v, &hm.idy_c, &hm.dy_c, &hm.dy_v, &hm.wx, &hm.wy};
    size_t mtot = 0;
    for (auto *v : mv) mtot += v->size();
    if (cudaMalloc(&c->metric_mem, mtot * sizeof(double)) != cudaSuccess) return fail(PVOF_ENOMEM, "cudaMalloc metrics");
    std::vector<double> mh;
    mh.reserve(mtot);
    std::vector<const double *> mptr;
    for (auto *v : mv) {
        mptr.push_back(c->metric_mem + mh.size() + NG);
        mh.insert(mh.end(), v->begin(), v->end());
    }
    if (cudaMemcpy(c->metric_mem, mh.data(), mtot * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(PVOF_ECUDA, "metric copy");
    d.m.idx_u = mptr[0]; d.m.idx_c = mptr[1]; d.m.dx_c = mptr[2]; d.m.dx_u = mptr[3];
    d.m.r_u = mptr[4]; d.m.r_c = mptr[5]; d.m.inv_r_u = mptr[6]; d.m.inv_r_c = mptr[7]; d.m.ring_wt_c = mptr[8];
    d.m.idy_v = mptr[9]; d.m.idy_c = mptr[10]; d.m.dy_c = mptr[11]; d.m.dy_v = mptr[12];
    d.m.wx = mptr[13]; d.m.wy = mptr[14];
    // ghost maps
    std::vector<int> srcs;
    std::vector<double> muls;
    std::vector<size_t> offx(BK_COUNT), offy(BK_COUNT);
    bool axis_lo = d.axisym;
    std::vector<HostMap> hmaps(BK_COUNT);
    for (int k = 0; k < BK_COUNT; k++) {
        Map1 mx, my;
        axis_map(mx, k, d.NX, d.perx, grid->wall[PVOF_LEFT], grid->wall[PVOF_RIGHT], axis_lo, true, true);
        axis_map(my, k, d.NY, d.pery, grid->wall[PVOF_BOTTOM], grid->wall[PVOF_TOP], false, false, false);
        hmaps[k].xsrc = mx.src; hmaps[k].xmul = mx.mul;
        hmaps[k].ysrc = my.src; hmaps[k].ymul = my.mul;
        offx[k] = srcs.size();
        srcs.insert(srcs.end(), mx.src.begin(), mx.src.end());
        muls.insert(muls.end(), mx.mul.begin(), mx.mul.end());
        offy[k] = srcs.size();
        srcs.insert(srcs.end(), my.src.begin(), my.src.end());
        muls.insert(muls.end(), my.mul.begin(), my.mul.end());
    }
    if (cudaMalloc(&c->map_src_mem, srcs.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->map_mul_mem, muls.size() * sizeof(double)) != cudaSuccess)
        return fail(PVOF_ENOMEM, "cudaMalloc maps");
    cudaMemcpy(c->map_src_mem, srcs.data(), srcs.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(c->map_mul_mem, muls.data(), muls.size() * sizeof(double), cudaMemcpyHostToDevice);
    for (int k = 0; k < BK_COUNT; k++) {
        c->maps[k].x.src = c->map_src_mem + offx[k];
        c->maps[k].x.mul = c->map_mul_mem + offx[k];
        c->maps[k].y.src = c->map_src_mem + offy[k];
        c->maps[k].y.mul = c->map_mul_mem + offy[k];
    }
    // persistent-solver occupancy
    int nsm = 0, ob = 0, o1 = 0, o2 = 0, o3 = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (!coop) return fail(PVOF_ENODEV, "device without cooperative launch");
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_cg_biharmonic, COOP_THREADS, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_cg_velocity, COOP_THREADS, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3, k_cg_pressure_fw, COOP_THREADS, 0);
    {   // the two grid-wide pressure kernels take the same block count
        int o3p = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o3p, k_cg_pressure_fwp, COOP_THREADS, 0);
        o3 = std::min(o3, o3p);
    }
    ob = std::min(o1, std::min(o2, o3));
    if (ob < 1) return fail(PVOF_ECUDA, "persistent solver kernels do not fit on an SM");
    c->coop_blocks_of[PVOF_SOLVER_BIHARMONIC] = o1 * nsm;   // each as many as it keeps co-resident
    c->coop_blocks_of[PVOF_SOLVER_VELOCITY] = o2 * nsm;
    c->coop_blocks_of[PVOF_SOLVER_PRESSURE] = o3 * nsm;
    c->coop_blocks = std::max(o1, std::max(o2, o3)) * nsm;
    c->coop_threads = COOP_THREADS;
    // cluster-resident solvers when the solve ranges fit one cluster
    // (pvof_set_cluster_solvers selects the grid-wide forms instead)
    {
        c->cgs_p_fit = cgs_pressure_setup(d.NX, d.NY, d.axisym, hmaps[BK_PRESSURE]);
        c->cgs_p_smem = c->cgs_p_fit.smem;
        c->cgs_p_threads = c->cgs_p_fit.threads;
        int ru[4], rv[4];
        u_range(c, ru[0], ru[1], ru[2], ru[3]);
        v_range(c, rv[0], rv[1], rv[2], rv[3]);
        c->cgs_v_fit = cgs_velocity_setup(ru, hmaps[BK_U_CG], rv, hmaps[BK_V_CG], d.axisym);
        c->cgs_v_smem = c->cgs_v_fit.smem;
        c->cgs_v_threads = c->cgs_v_fit.threads;
    }
    size_t npart = 4 * (size_t)std::max(c->coop_blocks, (int)(((d.NX + TBX - 1) / TBX) * ((d.NY + TBY - 1) / TBY)));
    if (cudaMalloc(&c->partials, npart * sizeof(double)) != cudaSuccess) return fail(PVOF_ENOMEM, "cudaMalloc partials");
    if (cudaMalloc(&c->scal, sizeof(DevScalars)) != cudaSuccess) return fail(PVOF_ENOMEM, "cudaMalloc scalars");
    cudaMemset(c->scal, 0, sizeof(DevScalars));
    if (cudaMallocHost(&c->scal_host, sizeof(DevScalars)) != cudaSuccess) return fail(PVOF_ENOMEM, "pinned scalars");
    std::memset(c->scal_host, 0, sizeof(DevScalars));
    for (int q = 0; q < 2; q++)
        if (cudaEventCreate(&c->timer_ev[q]) != cudaSuccess) return fail(PVOF_ECUDA, "event create");
    for (int q = 0; q < Ctx::NPEND; q++)
        for (int e = 0; e < 2; e++)
            if (cudaEventCreate(&c->pend_ev[q][e]) != cudaSuccess) return fail(PVOF_ECUDA, "event create");
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(PVOF_ECUDA, "create sync");
    c->stage = 0;
    c->dt = 0.0;
    *out = c;
    return PVOF_OK;
}

int pvof_destroy(pvof_ctx *c)
{
    if (!c) return PVOF_OK;
    if (c->h3) {
        pvof3::destroy(c->h3);
        delete c;
        return PVOF_OK;
    }
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int q = 0; q < PVOF_F_COUNT; q++) if (c->base[q]) cudaFree(c->base[q]);
    for (int q = 0; q < SC_COUNT; q++) if (c->sbase[q]) cudaFree(c->sbase[q]);
    if (c->metric_mem) cudaFree(c->metric_mem);
    if (c->map_src_mem) cudaFree(c->map_src_mem);
    if (c->map_mul_mem) cudaFree(c->map_mul_mem);
    if (c->partials) cudaFree(c->partials);
    cudaFree(c->cnn_params);
    cudaFree(c->cnn_bf16);
    cudaFree(c->cnn_x);
    cudaFree(c->cnn_y);
    cudaFree(c->cnn_work);
    if (c->scal) cudaFree(c->scal);
    if (c->scal_host) cudaFreeHost(c->scal_host);
    if (c->flush_buf) cudaFree(c->flush_buf);
    if (c->host_stage) cudaFree(c->host_stage);
    for (int q = 0; q < 2; q++) if (c->timer_ev[q]) cudaEventDestroy(c->timer_ev[q]);
    for (int q = 0; q < Ctx::NPEND; q++)
        for (int e = 0; e < 2; e++) if (c->pend_ev[q][e]) cudaEventDestroy(c->pend_ev[q][e]);
    delete c->ibm;
    delete c->tune;
    advect_maps_destroy(c->adv_maps);
    for (GraphEntry &g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->fft_coef) cudaFree(c->fft_coef);
    if (c->spec_mem) cudaFree(c->spec_mem);
    if (c->spec_s) cudaFree(c->spec_s);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PVOF_OK;
}

size_t pvof_field_block_count(const pvof_ctx *c, int field)
{
    if (!c || field < 0 || field >= PVOF_F_COUNT) return 0;
    if (c->h3) return pvof3::block_count(c->h3, field);
    size_t NX = (size_t)c->dom.NX, NY = (size_t)c->dom.NY, NZ = (size_t)c->g.NZM + 1;
    if (is_ng(field)) return NX * NY * NZ;
    return (NX + 2 * NG) * (NY + 2 * NG) * (NZ + 2 * NG);
}

// the device staging block of the host copies (one field's plane, grown on demand)
static int host_stage(pvof_ctx *c, size_t elems)
{
    if (c->host_stage_elems >= elems) return PVOF_OK;
    CK(cudaStreamSynchronize(c->stream));   // the old block may be in use
    cudaFree(c->host_stage);
    c->host_stage = nullptr;
    c->host_stage_elems = 0;
    if (cudaMalloc(&c->host_stage, elems * sizeof(double)) != cudaSuccess)
        return set_err(PVOF_ENOMEM, "cudaMalloc host staging block");
    c->host_stage_elems = elems;
    return PVOF_OK;
}

// One field between its host block (the reference's layout) and the device
// plane: one contiguous copy of the k = 0 plane (the 2D modes keep the k
// planes identical) through a staging block, the row pitch done by a kernel
// (a pitched 2D copy moves each short row as its own transfer).
int pvof_upload_field(pvof_ctx *c, int field, const double *host, size_t count)
{
    if (!c || !host) return set_err(PVOF_EINVAL, "null argument");
    if (c->h3) return from3(pvof3::upload(c->h3, field, host, count));
    if (count != pvof_field_block_count(c, field)) return set_err(PVOF_EINVAL, "block size does not match the field");
    CK(cudaSetDevice(c->device));
    const size_t NX = (size_t)c->dom.NX, NY = (size_t)c->dom.NY;
    const bool ng = is_ng(field);
    const size_t W = ng ? NX : NX + 2 * NG, H = ng ? NY : NY + 2 * NG;
    const double *plane = ng ? host : host + (size_t)NG * W * H;   // k = 0
    double *dst = ng ? c->f[field] : c->f[field] - (ptrdiff_t)NG * c->dom.P - NG;
    TRY(host_stage(c, W * H));
    CK(cudaMemcpyAsync(c->host_stage, plane, W * H * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_unpack_rows<<<(unsigned)((W * H + 255) / 256), 256, 0, c->stream>>>(dst, c->dom.P, c->host_stage, (int)W, (int)H);
    CKL(c);
    return PVOF_OK;
}

int pvof_download_field(pvof_ctx *c, int field, double *host, size_t count)
{
    if (!c || !host) return set_err(PVOF_EINVAL, "null argument");
    if (c->h3) return from3(pvof3::download(c->h3, field, host, count));
    if (count != pvof_field_block_count(c, field)) return set_err(PVOF_EINVAL, "block size does not match the field");
    CK(cudaSetDevice(c->device));
    const size_t NX = (size_t)c->dom.NX, NY = (size_t)c->dom.NY, NZ = (size_t)c->g.NZM + 1;
    const bool ng = is_ng(field);
    const size_t W = ng ? NX : NX + 2 * NG, H = ng ? NY : NY + 2 * NG;
    const double *src = ng ? c->f[field] : c->f[field] - (ptrdiff_t)NG * c->dom.P - NG;
    TRY(host_stage(c, W * H));
    k_pack_rows<<<(unsigned)((W * H + 255) / 256), 256, 0, c->stream>>>(c->host_stage, src, c->dom.P, (int)W, (int)H);
    CKL(c);
    for (size_t k = 0; k < NZ; k++)
        CK(cudaMemcpyAsync(host + (ng ? k : NG + k) * W * H, c->host_stage, W * H * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PVOF_OK;
}

int pvof_synchronize(pvof_ctx *c)
{
    if (!c) return set_err(PVOF_EINVAL, "null context");
    if (c->h3) return from3(pvof3::synchronize(c->h3));
    CK(cudaStreamSynchronize(c->stream));
    return PVOF_OK;
}

int pvof_set_stage(pvof_ctx *c, int which_stage, double dt)
{
    if (!c) return set_err(PVOF_EINVAL, "null context");
    if (which_stage < 0 || which_stage > 2 || !(dt > 0.0)) return set_err(PVOF_EINVAL, "stage must be 0..2 and dt > 0");
    if (c->h3) return from3(pvof3::set_stage(c->h3, which_stage, dt));
    c->stage = which_stage;
    c->dt = dt;
    return PVOF_OK;
}

#define ENTER(c)                                                        \
    do {                                                                \
        if (!(c)) return set_err(PVOF_EINVAL, "null context");          \
        if ((c)->h3) return set_err(PVOF_EINVAL, "not available in the 3D mode"); \
        CK(cudaSetDevice((c)->device));                                 \
    } while (0)
// entry points that the 3D mode supports: null check only
#define ENTER_ANY(c)                                                    \
    do {                                                                \
        if (!(c)) return set_err(PVOF_EINVAL, "null context");          \
    } while (0)
#define NEED_DT(c)                                                      \
    do {                                                                \
        if (!((c)->dt > 0.0)) return set_err(PVOF_EINVAL, "pvof_set_stage() first"); \
    } while (0)

int pvof_initialize(pvof_ctx *c)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::initialize(c->h3));
    ENTER(c);
    return initialize(c);
}
int pvof_VOF_DIFFUSE_init(pvof_ctx *c) { ENTER(c); return vof_diffuse_init(c); }
int pvof_VOF_DIFFUSE_step(pvof_ctx *c, pvof_stats *st)
{
    ENTER(c);
    NEED_DT(c);
    TRY(vof_diffuse_step(c));
    TRY(read_scalars(c));
    fill_stats(c, st);
    return PVOF_OK;
}
int pvof_VOF_DIFFUSE_advect_WENO5(pvof_ctx *c) { ENTER(c); return advect(c, F(c, PVOF_F_CH_RHS_CUR)); }
int pvof_VOF_update_density_viscosity(pvof_ctx *c) { ENTER(c); return update_density_viscosity(c); }
int pvof_VOF_DIFFUSE_compute_psi_LG(pvof_ctx *c) { ENTER(c); return compute_psi_LG(c); }
int pvof_VOF_DIFFUSE_compute_f_sigma(pvof_ctx *c) { ENTER(c); return compute_f_sigma(c); }
int pvof_VOF_apply_f_sigma_old(pvof_ctx *c) { ENTER(c); return apply_f_sigma_old(c); }
int pvof_VOF_swap_f_sigma(pvof_ctx *c) { ENTER(c); swap_f_sigma(c); return PVOF_OK; }
int pvof_Velocity_add_gravity_2_RHS(pvof_ctx *c) { ENTER(c); return add_gravity(c); }
int pvof_Velocity_cell_center(pvof_ctx *c) { ENTER(c); return cell_center(c); }

static int comp_of(char c) { return c == 'u' ? 0 : (c == 'v' ? 1 : -1); }

int pvof_Velocity_set_implicit_explicit(pvof_ctx *c, char component)
{
    ENTER(c);
    int k = comp_of(component);
    if (k < 0) return set_err(PVOF_EINVAL, "component must be 'u' or 'v' in the 2D modes");
    return implicit_explicit(c, k);
}
int pvof_Velocity_set_RHS(pvof_ctx *c, char component)
{
    ENTER(c);
    NEED_DT(c);
    int k = comp_of(component);
    if (k < 0) return set_err(PVOF_EINVAL, "component must be 'u' or 'v' in the 2D modes");
    return set_rhs(c, k);
}
int pvof_Velocity_solve_cg(pvof_ctx *c, char component, pvof_stats *st)
{
    ENTER(c);
    NEED_DT(c);
    int k = comp_of(component);
    if (k < 0) return set_err(PVOF_EINVAL, "component must be 'u' or 'v' in the 2D modes");
    TRY(velocity_solve(c, k));
    TRY(read_scalars(c));
    fill_stats(c, st);
    return c->scal_host->vel_iters[k];
}
int pvof_Velocity_update_boundaries(pvof_ctx *c, char component)
{
    ENTER(c);
    int k = comp_of(component);
    if (k < 0) return set_err(PVOF_EINVAL, "component must be 'u' or 'v' in the 2D modes");
    return fill(c, k == 0 ? BK_U : BK_V, F(c, k == 0 ? PVOF_F_U : PVOF_F_V));
}
int pvof_Pressure_set_RHS(pvof_ctx *c) { ENTER(c); NEED_DT(c); return p_set_rhs(c); }
int pvof_Pressure_compute_preconditioner(pvof_ctx *c) { ENTER(c); return p_precond(c); }
int pvof_Pressure_solve_cg(pvof_ctx *c, pvof_stats *st)
{
    ENTER(c);
    TRY(p_solve(c));
    TRY(read_scalars(c));
    fill_stats(c, st);
    return c->scal_host->p_iters;
}
int pvof_Pressure_project_velocity(pvof_ctx *c) { ENTER(c); NEED_DT(c); return p_project(c); }
int pvof_Pressure_compute_velocity_divergence(pvof_ctx *c, double *div_max)
{
    ENTER(c);
    TRY(p_divergence_async(c));
    TRY(read_scalars(c));
    if (div_max) *div_max = c->scal_host->div_max;
    return PVOF_OK;
}

int pvof_substep(pvof_ctx *c, pvof_stats *st)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::substep(c->h3, st));
    ENTER(c);
    NEED_DT(c);
    return substep(c, st);
}

int pvof_run_steps(pvof_ctx *c, int nsteps, double dt, pvof_stats *st)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::run_steps(c->h3, nsteps, dt, st));
    ENTER(c);
    if (nsteps < 0 || !(dt > 0.0)) return set_err(PVOF_EINVAL, "nsteps >= 0 and dt > 0");
    for (int n = 0; n < nsteps; n++) {
        for (int rk = 0; rk < 3; rk++) {
            if (c->time != 0 && rk == 0) TRY(cell_center(c));
            c->stage = rk;
            c->dt = dt;
            TRY(substep(c, st));
            c->time += dt * bet2(rk);
        }
    }
    return PVOF_OK;
}

int pvof_run_steps_batched(pvof_ctx *const *ctxs, int n, int nsteps, double dt, pvof_stats *stats)
{
    if (n < 0 || (n > 0 && !ctxs)) return set_err(PVOF_EINVAL, "bad context array");
    for (int q = 0; q < n; q++) {
        if (!ctxs[q]) return set_err(PVOF_EINVAL, "null context in the batch");
        if (ctxs[q]->h3) return set_err(PVOF_EINVAL, "the batched form takes 2D contexts");
        for (int r = 0; r < q; r++)
            if (ctxs[r] == ctxs[q]) return set_err(PVOF_EINVAL, "a context appears twice in the batch");
    }
    // with several cases on the GPU each case's momentum solve takes one
    // cluster (u, then v) instead of two side by side, so more cases fit
    const bool one = n > 1;
    std::vector<int> saved((size_t)n);
    for (int q = 0; q < n; q++) {
        saved[(size_t)q] = ctxs[q]->vel_one_cluster;
        ctxs[q]->vel_one_cluster = one ? 1 : saved[(size_t)q];
    }
    std::vector<int> rc((size_t)n, PVOF_OK);
    std::vector<std::string> msg((size_t)n);
    std::vector<std::thread> workers;
    workers.reserve((size_t)n);
    for (int q = 0; q < n; q++)
        workers.emplace_back([&, q]() {
            rc[(size_t)q] = pvof_run_steps(ctxs[q], nsteps, dt, stats ? &stats[q] : nullptr);
            if (rc[(size_t)q] < 0) msg[(size_t)q] = g_err;   // the message is per thread
        });
    for (std::thread &t : workers) t.join();
    for (int q = 0; q < n; q++) ctxs[q]->vel_one_cluster = saved[(size_t)q];
    for (int q = 0; q < n; q++)
        if (rc[(size_t)q] < 0) return set_err(rc[(size_t)q], "case " + std::to_string(q) + ": " + msg[(size_t)q]);
    return PVOF_OK;
}

int pvof_liquid_mass(pvof_ctx *c, double *mass)
{
    ENTER_ANY(c);
    if (c->h3) {
        double m = 0.0;
        const int rc = from3(pvof3::liquid_mass(c->h3, &m));
        if (mass) *mass = m;
        return rc;
    }
    ENTER(c);
    const int NX = c->dom.NX, NY = c->dom.NY;
    dim3 blk(TBX, TBY);
    dim3 grd((unsigned)((NX - 1 + TBX - 1) / TBX), (unsigned)((NY - 1 + TBY - 1) / TBY));
    k_mass<<<grd, blk, 0, c->stream>>>(c->dom, 0, NX - 1, 0, NY - 1, F(c, PVOF_F_C_L), c->partials);
    CKL(c);
    k_finalize_sum<<<1, 256, 0, c->stream>>>(c->partials, (int)(grd.x * grd.y), &c->scal->mass);
    CKL(c);
    TRY(read_scalars(c));
    if (mass) *mass = c->scal_host->mass;
    return PVOF_OK;
}

long long pvof_launch_count(const pvof_ctx *c) { return c ? (c->h3 ? pvof3::launch_count(c->h3) : c->launches) : 0; }

int pvof_timer_start(pvof_ctx *c)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::timer_start(c->h3));
    ENTER(c);
    CK(cudaEventRecord(c->timer_ev[0], c->stream));
    return PVOF_OK;
}

int pvof_timer_stop(pvof_ctx *c, double *ms)
{
    ENTER_ANY(c);
    if (c->h3) {
        double t = 0.0;
        const int rc = from3(pvof3::timer_stop(c->h3, &t));
        if (ms) *ms = t;
        return rc;
    }
    ENTER(c);
    CK(cudaEventRecord(c->timer_ev[1], c->stream));
    CK(cudaEventSynchronize(c->timer_ev[1]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->timer_ev[0], c->timer_ev[1]));
    if (ms) *ms = t;
    return PVOF_OK;
}

int pvof_flush_l2(pvof_ctx *c)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::flush_l2(c->h3));
    ENTER(c);
    if (!c->flush_buf) {
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device);
        c->flush_bytes = (size_t)std::max(l2, 1 << 20) * 2;
        if (cudaMalloc(&c->flush_buf, c->flush_bytes) != cudaSuccess) {
            c->flush_buf = nullptr;
            return set_err(PVOF_ENOMEM, "cudaMalloc flush buffer");
        }
    }
    CK(cudaMemsetAsync(c->flush_buf, (int)(c->launches & 0xff), c->flush_bytes, c->stream));
    return PVOF_OK;
}

int pvof_set_graphs(pvof_ctx *c, int enabled)
{
    ENTER(c);
    c->use_graphs = enabled ? 1 : 0;
    return PVOF_OK;
}

long long pvof_graph_replays(const pvof_ctx *c) { return (c && !c->h3) ? c->graph_replays : -1; }

int pvof_clamp_mass_total(const pvof_ctx *c, double *total)
{
    if (!c || !total) return set_err(PVOF_EINVAL, "null context or output");
    *total = c->h3 ? pvof3::clamp_total(c->h3) : c->clamp_total;
    return PVOF_OK;
}

int pvof_set_pressure_pairs(pvof_ctx *c, int mode)
{
    ENTER(c);
    if (mode < -1 || mode > 1) return set_err(PVOF_EINVAL, "pvof_set_pressure_pairs: mode -1, 0 or 1");
    // the captured substeps hold the old solver launches: wait for them and drop them
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->pressure_pairs = mode;
    return PVOF_OK;
}

int pvof_set_cluster_solvers(pvof_ctx *c, int enabled)
{
    ENTER(c);
    // the captured substeps hold the old solver launches: wait for them and drop them
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    const StripPlan none = {0, 0};
    const StripPlan &pp = enabled ? c->cgs_p_fit : none;
    const StripPlan &vp = enabled ? c->cgs_v_fit : none;
    c->cgs_p_smem = pp.smem;
    c->cgs_p_threads = pp.threads;
    c->cgs_v_smem = vp.smem;
    c->cgs_v_threads = vp.threads;
    return PVOF_OK;
}

long long pvof_spectral_tables(int N, int M, double idx2, double idy2, double *out, long long cap)
{
    int odd = N;
    while (odd % 2 == 0 && odd > 1) odd /= 2;
    if (N < 2 || N % 2 != 0 || (odd != 1 && odd != 3 && odd != 5) || M < 2 || !(idx2 > 0.0) || !(idy2 > 0.0)) {
        set_err(PVOF_EINVAL, "pvof_spectral_tables: N = 2^a, 3 2^a or 5 2^a (even), M >= 2, positive spacings");
        return -1;
    }
    std::vector<double> tw, tri;
    spec_tables(N, M, idx2, idy2, tw, tri);
    const long long n = (long long)tri.size();
    if (out && cap >= n) std::memcpy(out, tri.data(), tri.size() * sizeof(double));
    return n;
}

int pvof_set_autotune(pvof_ctx *c, int enabled)
{
    ENTER(c);
    drop_graphs(c);   // they hold the launches' tiles
    if (!c->tune) {
        c->tune = new TuneState();
        bool ok = true;
        for (int q = 0; q < TUNE_EVENTS && ok; q++)
            ok = cudaEventCreate(&c->tune->ev[q][0]) == cudaSuccess && cudaEventCreate(&c->tune->ev[q][1]) == cudaSuccess;
        if (!ok) {
            delete c->tune;
    advect_maps_destroy(c->adv_maps);
            c->tune = nullptr;
            return set_err(PVOF_ECUDA, "cudaEventCreate for the autotuner");
        }
        c->tune->events = true;
    }
    c->tune->recs.clear();
    c->tune->npend = 0;
    c->tune->active = enabled != 0;
    return PVOF_OK;
}

int pvof_autotune_active(const pvof_ctx *c) { return c && c->tune && c->tune->active ? 1 : 0; }

int pvof_autotune_entries(const pvof_ctx *c) { return c && c->tune ? (int)c->tune->recs.size() : 0; }

int pvof_autotune_entry(const pvof_ctx *c, int q, const char **name, int *bx, int *by, double *best_ms,
                        double *default_ms)
{
    if (!c || !c->tune || q < 0 || q >= (int)c->tune->recs.size()) return set_err(PVOF_EINVAL, "bad autotuner entry");
    const TuneRec &r = c->tune->recs[(size_t)q];
    if (name) *name = r.name;
    const int k = r.chosen >= 0 ? r.chosen : 0;
    if (bx) *bx = TUNE_TILES[k].bx;
    if (by) *by = TUNE_TILES[k].by;
    if (best_ms) *best_ms = r.n[k] ? r.ms[k] / r.n[k] : 0.0;
    if (default_ms) *default_ms = r.n[0] ? r.ms[0] / r.n[0] : 0.0;
    return r.chosen >= 0 ? 1 : 0;
}

int pvof_set_solver_timing(pvof_ctx *c, int enabled)
{
    ENTER_ANY(c);
    if (c->h3) return from3(pvof3::set_solver_timing(c->h3, enabled));
    ENTER(c);
    c->solver_timing = enabled ? 1 : 0;
    for (int k = 0; k < 3; k++) {
        c->sol_ms[k] = 0.0;
        c->sol_launches[k] = c->sol_iters[k] = c->sol_cell_iters[k] = 0;
    }
    c->npend = 0;
    return PVOF_OK;
}

const char *pvof_solver_kernel(const pvof_ctx *c, int solver)
{
    if (!c) return "";
    if (c->h3) {
        static const char *k3[] = {"k3_reduce (biharmonic CG)", "k3_reduce (velocity PCG)", "k3_reduce (pressure PCG)"};
        return (solver >= 0 && solver <= 2) ? k3[solver] : "";
    }
    switch (solver) {
    case PVOF_SOLVER_BIHARMONIC: return "k_cg_biharmonic";
    case PVOF_SOLVER_VELOCITY: return c->cgs_v_smem ? "k_cgs_velocity" : "k_cg_velocity";
    case PVOF_SOLVER_PRESSURE:
        return c->cgs_p_smem ? "k_cgs_pressure" : (grid_pressure_pairs(c) ? "k_cg_pressure_fwp" : "k_cg_pressure_fw");
    default: return "";
    }
}

int pvof_solver_timing(const pvof_ctx *c, int solver, double *ms, long long *launches, long long *iterations,
                       long long *cell_iters)
{
    if (!c || solver < 0 || solver > 2) return set_err(PVOF_EINVAL, "bad solver index");
    if (c->h3) return from3(pvof3::solver_timing(c->h3, solver, ms, launches, iterations, cell_iters));
    if (ms) *ms = c->sol_ms[solver];
    if (launches) *launches = c->sol_launches[solver];
    if (iterations) *iterations = c->sol_iters[solver];
    if (cell_iters) *cell_iters = c->sol_cell_iters[solver];
    return PVOF_OK;
}


// --- resolved solid particles --------------------------------------------
int pvof_set_particles(pvof_ctx *c, const pvof_particle *parts, int n)
{
    ENTER(c);
    if (n < 0 || (n > 0 && !parts)) return set_err(PVOF_EINVAL, "bad particle array");
    for (int q = 0; q < n; q++) {
        if (!(parts[q].R > 0.0)) return set_err(PVOF_EINVAL, "particle radius must be positive");
        // Lagrangian_generate_points_2d (Lagrangian.c:2948-2959): axisymmetric
        // particles are spheres centred on the axis
        if (c->dom.axisym && std::fabs(parts[q].X[0]) > 1.0e-14)
            return set_err(PVOF_EINVAL, "an axisymmetric particle must sit on the axis (X[0] = 0)");
    }
    IbmState *s;
    TRY(ibm_state(c, &s));
    CK(cudaStreamSynchronize(c->stream));   // the buffers below may be in use
    PGrid &g = s->P.g;
    g.Cn = c->p.Cn;
    for (int k = 0; k < 3; k++) g.grav[k] = c->p.grav[k];
    std::vector<PEnt> mob, fix;
    for (int q = 0; q < n; q++) {
        const pvof_particle &p = parts[q];
        PEnt e;
        std::memset(&e, 0, sizeof(e));
        e.X[0] = p.X[0];
        e.X[1] = p.X[1];
        e.R = p.R;
        e.U[0] = p.U[0];
        e.U[1] = p.U[1];
        e.Omega[2] = p.Omega_z;
        e.rho_s = p.rho_s;
        (p.mobile ? mob : fix).push_back(e);
    }
    // IDs as Particle_initialize gives them: fixed first, then mobile (Particle.c:213-221)
    int id = 0;
    for (PEnt &e : fix) e.id = id++;
    for (PEnt &e : mob) e.id = id++;
    std::vector<const PEnt *> by_id(n);
    for (PEnt &e : fix) by_id[e.id] = &e;
    for (PEnt &e : mob) by_id[e.id] = &e;
    for (PEnt &e : mob) { e.mobile = 1; ps_derived(e, g); }
    for (PEnt &e : fix) { e.mobile = 0; ps_derived(e, g); }
    std::vector<double> trig;
    std::vector<int> trig_off(n > 0 ? n : 1, 0);
    long long nl = 0;
    for (int q = 0; q < n; q++) {
        trig_off[q] = (int)nl;
        ps_marker_table(*by_id[q], g, trig);
        nl += by_id[q]->N_L;
    }
    // capacities: a particle has at most two copies per periodic axis, so at
    // most nine entries; markers likewise
    PSet &P = s->P;
    P.cap_own = n > 0 ? n : 1;
    P.cap_ent = 9 * P.cap_own;
    P.cap_mk = (int)std::max(9 * nl, 1LL);
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t o_mob = take(sizeof(PEnt) * P.cap_own), o_fix = take(sizeof(PEnt) * P.cap_own);
    const size_t o_ent = take(sizeof(PEnt) * P.cap_ent), o_tmp = take(sizeof(PEnt) * 3 * (size_t)P.cap_ent);
    const size_t o_dent = take(sizeof(IbmEntryDev) * P.cap_ent);
    const size_t o_mk = take(sizeof(double) * 6 * (size_t)P.cap_mk), o_flag = take(sizeof(int) * 4 * (size_t)P.cap_mk);
    const size_t o_trig = take(sizeof(double) * std::max<size_t>(trig.size(), 1));
    const size_t o_toff = take(sizeof(int) * trig_off.size());
    const size_t o_plist = take(sizeof(double) * 4 * (size_t)P.cap_ent);
    const size_t o_geo = take(sizeof(double) * 3 * (size_t)P.cap_own);
    const size_t o_FT = take(sizeof(double) * 6 * (size_t)P.cap_ent), o_sums = take(sizeof(double) * 6 * (size_t)P.cap_ent);
    cudaFree(s->d_mem);
    s->d_mem = nullptr;
    if (cudaMalloc(&s->d_mem, off) != cudaSuccess) return set_err(PVOF_ENOMEM, "cudaMalloc particle state");
    char *m = s->d_mem;
    P.mob = (PEnt *)(m + o_mob);
    P.fix = (PEnt *)(m + o_fix);
    P.ent = (PEnt *)(m + o_ent);
    P.tmp = (PEnt *)(m + o_tmp);
    P.dent = (IbmEntryDev *)(m + o_dent);
    P.mk = (double *)(m + o_mk);
    P.mflag = (int *)(m + o_flag);
    P.trig = (const double *)(m + o_trig);
    P.trig_off = (const int *)(m + o_toff);
    P.plist = (double *)(m + o_plist);
    P.geo = (double *)(m + o_geo);
    P.FT = (double *)(m + o_FT);
    P.sums = (double *)(m + o_sums);
    P.nmob = (int)mob.size();
    P.nfix = (int)fix.size();
    P.ne = P.nm = P.ngeo = P.err = 0;
    P.err_a = P.err_b = -1;
    // the contact-line list before the first update: the owned lists
    std::vector<double> pl;
    for (const std::vector<PEnt> *l : {&mob, &fix})
        for (const PEnt &e : *l) {
            pl.push_back(e.X[0]);
            pl.push_back(e.X[1]);
            pl.push_back(e.R);
            pl.push_back((double)e.id);
        }
    P.np = n;
    CK(cudaMemsetAsync(s->d_mem, 0, off, c->stream));
    if (!mob.empty()) CK(cudaMemcpyAsync(P.mob, mob.data(), mob.size() * sizeof(PEnt), cudaMemcpyHostToDevice, c->stream));
    if (!fix.empty()) CK(cudaMemcpyAsync(P.fix, fix.data(), fix.size() * sizeof(PEnt), cudaMemcpyHostToDevice, c->stream));
    if (!trig.empty())
        CK(cudaMemcpyAsync((void *)P.trig, trig.data(), trig.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync((void *)P.trig_off, trig_off.data(), trig_off.size() * sizeof(int), cudaMemcpyHostToDevice,
                       c->stream));
    if (!pl.empty()) CK(cudaMemcpyAsync(P.plist, pl.data(), pl.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(s->d_ps, &P, sizeof(PSet), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));   // the host vectors are released on return
    s->flagged = false;
    drop_graphs(c);
    return PVOF_OK;
}

int pvof_Lagrangian_flag_points(pvof_ctx *c) { ENTER(c); return ibm_flag_points(c); }

int pvof_particle_entries(pvof_ctx *c)
{
    ENTER(c);
    if (!c->ibm || !c->ibm->flagged) return set_err(PVOF_EINVAL, "pvof_Lagrangian_flag_points() first");
    PSet h;
    TRY(ibm_read(c, c->ibm, h));
    return h.ne;
}

int pvof_particle_forces(pvof_ctx *c, double *Fo, double *To, int nmax)
{
    ENTER(c);
    IbmState *s = c->ibm;
    if (!s || !s->flagged) return set_err(PVOF_EINVAL, "pvof_Lagrangian_flag_points() first");
    PSet hs;
    TRY(ibm_read(c, s, hs));
    const int ne = hs.ne;
    if (nmax < ne || !Fo || !To) return set_err(PVOF_EINVAL, "force arrays too small");
    std::vector<double> h(6 * (size_t)ne);
    if (ne) CK(cudaMemcpyAsync(h.data(), s->P.FT, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int e = 0; e < ne; e++)
        for (int k = 0; k < 3; k++) {
            Fo[3 * e + k] = h[6 * e + k];
            To[3 * e + k] = h[6 * e + 3 + k];
        }
    return ne;
}

int pvof_particle_markers(pvof_ctx *c, int entry, double *x, double *y, double *vol, int *flag, int nmax)
{
    ENTER(c);
    IbmState *s = c->ibm;
    if (!s || !s->flagged) return set_err(PVOF_EINVAL, "pvof_Lagrangian_flag_points() first");
    PSet hs;
    TRY(ibm_read(c, s, hs));
    if (entry < 0 || entry >= hs.ne) return set_err(PVOF_EINVAL, "bad particle entry");
    PEnt e;
    CK(cudaMemcpy(&e, s->P.ent + entry, sizeof(PEnt), cudaMemcpyDeviceToHost));
    if (nmax < e.mcount) return set_err(PVOF_EINVAL, "marker arrays too small");
    const size_t cap = (size_t)s->P.cap_mk;
    if (e.mcount > 0) {
        if (x) CK(cudaMemcpy(x, s->P.mk + e.moff, e.mcount * sizeof(double), cudaMemcpyDeviceToHost));
        if (y) CK(cudaMemcpy(y, s->P.mk + cap + e.moff, e.mcount * sizeof(double), cudaMemcpyDeviceToHost));
        if (vol) CK(cudaMemcpy(vol, s->P.mk + 2 * cap + e.moff, e.mcount * sizeof(double), cudaMemcpyDeviceToHost));
        if (flag) CK(cudaMemcpy(flag, s->P.mflag + e.moff, e.mcount * sizeof(int), cudaMemcpyDeviceToHost));
    }
    return e.mcount;
}

int pvof_VOF_DIFFUSE_compute_C_S(pvof_ctx *c) { ENTER(c); return compute_C_S(c); }
int pvof_VOF_DIFFUSE_compute_solid_normals_MCL(pvof_ctx *c) { ENTER(c); return mcl_normals(c); }
int pvof_Particle_initialize_velocities(pvof_ctx *c)
{
    ENTER(c);
    if (!c->ibm) return set_err(PVOF_EINVAL, "pvof_set_particles() first");
    return ibm_velocity_init(c);
}
int pvof_Lagrangian_advect_particles(pvof_ctx *c)
{
    ENTER(c);
    NEED_DT(c);
    return ibm_advect(c);
}
int pvof_set_pressure_network(pvof_ctx *c, const float *params, size_t n)
{
    ENTER(c);
    if (!params || n != pvof_cnn_param_count()) return set_err(PVOF_EINVAL, "network parameter count mismatch");
    const int W = c->dom.NX - 1, H = c->dom.NY - 1;
    const size_t plane = (size_t)W * H;
    if (!c->cnn_params) {
        if (cudaMalloc(&c->cnn_params, n * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&c->cnn_bf16, n * sizeof(uint16_t)) != cudaSuccess ||
            cudaMalloc(&c->cnn_x, 3 * plane * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&c->cnn_y, plane * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&c->cnn_work, pvof_cnn_work_floats(H, W) * sizeof(float)) != cudaSuccess)
            return set_err(PVOF_ENOMEM, "cudaMalloc network buffers");
    }
    CK(cudaMemcpyAsync(c->cnn_params, params, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    const int rc = pvof_cnn_to_bf16(c->cnn_params, c->cnn_bf16, c->stream);
    if (rc != PVOF_OK) return set_err(rc, "network weights");
    CK(cudaStreamSynchronize(c->stream));
    return PVOF_OK;
}

int pvof_pressure_network_sample(pvof_ctx *c, int stage, float *x, float *t)
{
    ENTER(c);
    if (stage < 0 || stage > 2 || !x || !t) return set_err(PVOF_EINVAL, "bad stage or null buffer");
    if (!(c->phi_old_mask >> stage & 1)) return set_err(PVOF_EINVAL, "no two kept corrections for this stage yet");
    TRY(cnn_prepare(c, S(c, SC_PHI_OLD + stage), S(c, SC_PHI_PREV + stage), x, t));
    CK(cudaStreamSynchronize(c->stream));
    return PVOF_OK;
}

int pvof_get_particles(pvof_ctx *c, pvof_particle *out, int *ids, double *Fo, double *To, int nmax)
{
    ENTER(c);
    IbmState *s;
    TRY(ibm_need(c, &s));
    PSet h;
    TRY(ibm_read(c, s, h));
    const int n = h.nmob + h.nfix;
    if (nmax < n || (n > 0 && !out)) return set_err(PVOF_EINVAL, "particle array too small");
    std::vector<PEnt> mob(h.nmob), fix(h.nfix);
    if (h.nmob) CK(cudaMemcpy(mob.data(), s->P.mob, h.nmob * sizeof(PEnt), cudaMemcpyDeviceToHost));
    if (h.nfix) CK(cudaMemcpy(fix.data(), s->P.fix, h.nfix * sizeof(PEnt), cudaMemcpyDeviceToHost));
    int q = 0;
    for (const std::vector<PEnt> *l : {&mob, &fix})
        for (const PEnt &e : *l) {
            pvof_particle &p = out[q];
            p.mobile = l == &mob ? 1 : 0;
            p.X[0] = e.X[0];
            p.X[1] = e.X[1];
            p.R = e.R;
            p.U[0] = e.U[0];
            p.U[1] = e.U[1];
            p.Omega_z = e.Omega[2];
            p.rho_s = e.rho_s;
            if (ids) ids[q] = e.id;
            for (int k = 0; k < 3; k++) {
                if (Fo) Fo[3 * q + k] = e.F[k];
                if (To) To[3 * q + k] = e.T[k];
            }
            q++;
        }
    return n;
}
int pvof_VOF_DIFFUSE_apply_contact_angle(pvof_ctx *c) { ENTER(c); return apply_contact_angle(c); }
int pvof_VOF_DIFFUSE_extend_psi_LG_contact_angle(pvof_ctx *c) { ENTER(c); return extend_psi_LG(c); }

int pvof_Velocity_solve_explicit(pvof_ctx *c, char component)
{
    ENTER(c);
    NEED_DT(c);
    int k = comp_of(component);
    if (k < 0) return set_err(PVOF_EINVAL, "component must be 'u' or 'v' in the 2D modes");
    return vel_explicit(c, k);
}

int pvof_Lagrangian_force(pvof_ctx *c, int force_iter)
{
    ENTER(c);
    NEED_DT(c);
    return ibm_force(c, force_iter);
}


int pvof_Pressure_solve_fft(pvof_ctx *c) { ENTER(c); return p_solve_fft(c); }

}  // extern "C"
