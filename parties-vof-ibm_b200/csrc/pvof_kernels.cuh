// Kernel declarations shared by the routine kernels, the solvers and the
// host orchestration.
#pragma once

#include <string>
#include <vector>

#include "pvof_internal.cuh"

namespace pvof {

struct BihArgs {
    Dom d;
    BcMap msc;             // scalar ghost update of x, p and the Laplacian
    double *x;             // C_L (solution, updated in place)
    const double *b;       // rhs_vec
    double *r, *p1, *p2, *Ap, *aux;
    double a_dt, bih, tol;
    int maxit;
    double *partials;
    DevScalars *scal;
};

struct VelArgs {
    Dom d;
    BcMap mcg;             // VEL_TYPE_CG ghost update of the direction
    int comp;              // 0 = u, 1 = v
    int i0, i1, j0, j1;    // solve range
    double *x;             // velocity component (updated in place)
    const double *rhs, *rho, *mu;
    double *r, *dir, *dir2, *z, *Ad, *diag;
    double iRe, alpha_dt, in_tot, tol;
    double step_eps;       // added to the step-length and direction denominators (1e-14 in the reference)
    int maxit;
    double *partials;
    DevScalars *scal;
    double *ft = nullptr, *mc = nullptr;   // time-term and corner-viscosity planes (k_cg_velocity)
};

struct PresArgs {
    Dom d;
    BcMap mp;              // Pressure_apply_BCs + exchange
    double *phi;           // deltap
    const double *rhs, *rho, *M;
    double *res, *dir, *dir2, *z, *Ad;
    double tol;
    int maxit;
    double *partials;
    DevScalars *scal;
    double *bx = nullptr, *by = nullptr;   // face-weight planes (k_cg_pressure_fw)
};

// spectral-preconditioned pressure PCG (pvof_spec.cu)
struct SpecScal {
    unsigned arrivals;   // arrivals at the solve's grid barriers, zeroed before each launch
};

constexpr int SPEC_PT = 1024;        // threads per block of the cooperative solve

struct SpecArgs {
    Dom d;
    BcMap mp;                 // the pressure ghost rules
    double *phi;              // deltap
    const double *rhs, *rho, *MJ;
    double *res, *z, *Ad, *hat;
    const double2 *tw;        // exp(-2 pi i k / N), k < N / 2
    const double *tri;        // the tridiagonal phase's coefficients, one set per wave number (spec_tables)
    double *cx, *cy, *sm;     // per solve: x and y face coefficients of the operator, sqrt of the Jacobi weights
    int N, logN, M;           // x cells (R n), log2 n, y cells
    int R, n;                 // N = R n: R = 1, 3 or 5, n a power of two
    double fscale;            // dy^2 / N
    double tol;
    int maxit;
    double *part;             // per-block sums, three slots of gridDim entries
    SpecScal *s;
    DevScalars *scal;
};

// VOF_DIFFUSE_advect_WENO5 as one TMA-tiled kernel (pvof_advect.cu)
struct AdvectMaps;
AdvectMaps *advect_maps_create(const double *C_base, const double *u_base, const double *v_base, int P, int NY);
void advect_maps_destroy(AdvectMaps *a);
cudaError_t advect_tma_launch(const AdvectMaps *a, const Dom &d, const BcMap &mu, const BcMap &mv, const double *C,
                              const double *u, const double *v, int weno5, bool fp32, double *out, DevScalars *scal,
                              cudaStream_t st);

__global__ void k_unpack_rows(double *dst, int P, const double *src, int W, int H);
__global__ void k_pack_rows(double *dst, const double *src, int P, int W, int H);

// raise a kernel's dynamic shared memory limit to at least bytes (never lower it)
bool raise_dynamic_smem(const void *fn, size_t bytes);

bool spec_supported(const Dom &d, const char **why);
int spec_tables(int N, int M, double idx2, double idy2, std::vector<double> &tw, std::vector<double> &tri);
int spec_pcg_blocks(int device, int N, int M);
cudaError_t spec_launch_pcg(const SpecArgs &A, int blocks, double *d0, double *d1, cudaStream_t st);
const void *spec_pcg_kernel();   // k_spec_pcg, for marking graph nodes cooperative

__global__ void k_fill(Dom d, BcMap m, double *f);
__global__ void k_bulk_S_f(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *CS, double *bS);
__global__ void k_laplacian_f(Dom d, int i0, int i1, int j0, int j1, const double *in, double *out);
__global__ void k_psi_LG_f(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *lap, double *psi,
                           double cn2);
__global__ void k_f_sigma_f(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *CG,
                            const double *CS, const double *psi, double *fx, double *fy, double scale, int ui0,
                            int ui1, int uj1, int vj0, int vi1, int vj1);
__global__ void k_bulk_S(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *CS, double *bS);
__global__ void k_laplacian(Dom d, int i0, int i1, int j0, int j1, const double *in, double *out);
__global__ void k_div_by(Dom d, int i0, int i1, int j0, int j1, double *a, double s);
__global__ void k_add(Dom d, int i0, int i1, int j0, int j1, double *a, const double *b);
__global__ void k_sub_scaled(Dom d, int i0, int i1, int j0, int j1, double *a, const double *b, double s);
__global__ void k_rhs_vec(Dom d, int i0, int i1, int j0, int j1, double *vec, const double *CL, const double *cur,
                          const double *rn, double a_dt, int s);
__global__ void k_bound(Dom d, int i0, int i1, int j0, int j1, double *CL, const double *CS, double *CG, double *partials);
__global__ void k_finalize_sum(const double *partials, int n, double *out);
__global__ void k_phase_cache(size_t n, const double *CL, const double *CS, double *CG, double *F);
__global__ void k_clamp_from(size_t n, const double *F, double *CL);
__global__ void k_density(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *CS, const double *CG,
                          double *rho, double *mu, double rho_g, double mu_g);
__global__ void k_psi_LG(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *lap, double *psi, double cn2);
__global__ void k_f_sigma(Dom d, int i0, int i1, int j0, int j1, const double *CL, const double *CG, const double *CS,
                          const double *psi, double *fx, double *fy, double scale, int ui0, int ui1, int uj1, int vj0,
                          int vi1, int vj1);
__global__ void k_add_to(Dom d, int i0, int i1, int j0, int j1, double *rhs, const double *f);
__global__ void k_gravity(Dom d, int i0, int i1, int j0, int j1, const double *rho, double *rhs, int di, int dj,
                          double Ri, double g);
__global__ void k_cell_center(Dom d, int i0, int i1, int j0, int j1, const double *u, const double *v, double *ub, double *vb);
__global__ void k_u_impexp(Dom d, int i0, int i1, int j0, int j1, const double *u, const double *v, const double *ub,
                           const double *mu, double *ex, double *im, double *vx, double iRe);
__global__ void k_v_impexp(Dom d, int i0, int i1, int j0, int j1, const double *u, const double *v, const double *vb,
                           const double *mu, double *ex, double *im, double *vx, double iRe);
__global__ void k_set_rhs(Dom d, int i0, int i1, int j0, int j1, int comp, const double *data, const double *pd,
                          const double *rho, double *rhs, const double *ex, double *exo, const double *vx, double *vxo,
                          const double *im, double a_dt, int s, double dp_src, int resolved);
__global__ void k_p_rhs(Dom d, int i0, int i1, int j0, int j1, const double *u, const double *v, double *rhs, double ihdt);
__global__ void k_p_precond(Dom d, int i0, int i1, int j0, int j1, const double *rho, double *M);
__global__ void k_p_update(Dom d, int i0, int i1, int j0, int j1, double *pd, const double *dp);
__global__ void k_project(Dom d, int i0, int i1, int j0, int j1, int comp, double *vel, const double *dp,
                          const double *rho, double mdt);
__global__ void k_div_max(Dom d, int i0, int i1, int j0, int j1, const double *u, const double *v, unsigned long long *out);
__global__ void k_mass(Dom d, int i0, int i1, int j0, int j1, const double *CL, double *partials);

// Cluster-resident solvers (pvof_cgs.cu).  The setup functions return the
// shared memory a solve range needs after setting the kernel attributes, or 0
// when the range does not fit one cluster, its ghost maps do not have the
// shape the strip layout assumes, or the cluster cannot be scheduled.
constexpr int CGC_CTAS = 16;   // CTAs per cluster

// host copy of one ghost-update kind: entry [i + NG] for i in [-NG, N + NG)
struct HostMap {
    std::vector<int> xsrc, ysrc;
    std::vector<double> xmul, ymul;
};

// the two velocity components of one launch: cluster q solves c[q]
struct VelPair {
    VelArgs c[2];
};


StripPlan cgs_pressure_setup(int NX, int NY, int axisym, const HostMap &mp);
cudaError_t cgs_pressure_launch(const PresArgs &A, const StripPlan &plan, cudaStream_t stream);
// ranges {i0, i1, j0, j1} of u and v; one plan serves both
StripPlan cgs_velocity_setup(const int ru[4], const HostMap &mu, const int rv[4], const HostMap &mv, int axisym);
cudaError_t cgs_velocity_launch(const VelPair &V, int ncomp, const StripPlan &plan, cudaStream_t stream);

// ---------------------------------------------------------------------------
// resolved solid particles (pvof_ibm.cu)
// ---------------------------------------------------------------------------

// one entry of a particle list after the update of a substep (an owned
// particle or a periodic copy)
struct IbmEntryDev {
    double X[3], U[3], Omega[3], Zs;
    double R, id;
    int moff, mcount;
    int box[4];
    int mbox[2][4];           // cells of Interpolate_integrate_momentum_twod for u and v
};

// per-entry sums at the end of a substep (k_ibm_particle_sums): Int_U[0..1],
// Int_Omega[2], and with ccf the capillary contact force F_CCF[0..1], T_CCF[2]
struct IbmSumArgs {
    const IbmEntryDev *ent;
    const int *ne;                       // entries (device count; the launch covers the capacity)
    const double *U, *V, *CL, *CS;
    const double *xu, *xc, *yv, *yc;     // offset by NG
    const double *plist;                 // x, y, R, ID of the list entries
    const int *np;                       // their count (device)
    double h, slab, sigma, ct, st, support_width;
    int nk, ccf;
    int axisym;                          // ring measures, no in-plane spin
    double theta_span;
    double *out;                         // 6 doubles per entry
};

// parity of a quantity across the symmetry axis for the marker gathers and
// spreads (Interpolate.c:334-388): none (planar), odd (u faces), even
constexpr int IBM_AXIS_NONE = 0, IBM_AXIS_ODD = 1, IBM_AXIS_EVEN = 2;

struct IbmDev {
    const IbmEntryDev *ent;
    const int *ne;                 // entries (device count; the launches cover the capacity)
    const double *XL, *YL, *vol;
    const int *flag;
    int *sup_i, *sup_j;            // lower corner of each marker's spreading support
    double *UL, *rhoL, *FL, *FT;   // FT: F[3], T[3] per entry
    double xlo, xhi, ylo, yhi;     // Lagrangian_local_point_2d bounds
    double h, dxu1, slab;
    const double *dyv;
    int axisym;                    // fold supports across the axis, ring cell volumes
    double theta_span;
};

void ibm_solid_constants(double cn, double &shift, double &denom, double &extra);

// contact-line projection (pvof_mcl.cu): the G-range scalars of one pass and
// the case constants; CL and field are the pass's snapshots
struct MclView {
    int NX, NY;
    int perx, pery;
    int free_lo_x, free_hi_x, free_lo_y, free_hi_y;   // free-slip walls (mirror maps)
    const double *xc, *yc;                            // offset by NG, valid on [-NG, N + NG)
    double ct, st;                                    // cos, sin of the contact angle
    int hydrophilic;                                  // theta <= pi / 2
    double cmin, cmax;                                // liquid-gas band
    const double *CS, *CG, *CL, *field;
};

__global__ void k_mcl_normals(Dom d, const double *xc, const double *yc, const double *CS, const double *plist,
                              const int *np, double support_width, double *nxo, double *nyo);
__global__ void k_mcl_apply(Dom d, MclView v, const double *nxa, const double *nya, double *CLout);
__global__ void k_mcl_axis_normals(Dom d, double *nx, double *ny);
__global__ void k_mcl_extend_psi(Dom d, MclView v, const double *nxa, const double *nya, double *PSIout);

__global__ void k_ibm_interp(Dom d, const double *a, const double *xs, const double *ys, double h, const double *XL,
                             const double *YL, const int *nm, int axis, double *out);
constexpr int IBM_FORCE_THREADS = 256;
__global__ void k_ibm_marker_force(IbmDev D, int comp, double xs0, double ys0, double idt2beta, int reset);
__global__ void k_ibm_spread(Dom d, IbmDev D, int comp, const double *xs, const double *ys, const double *rho,
                             double *rhs);
__global__ void k_ibm_correct(Dom d, int comp, double dtbeta, const double *rhs, const double *rho, double *vel);
__global__ void k_ibm_ng_update(Dom d, double *a, const double *b, int reset);
__global__ void k_vel_explicit(Dom d, int comp, int i0, int i1, int j0, int j1, double dtimeb, const double *rhs,
                               const double *rho, double *vel);
__global__ void k_ibm_particle_sums(Dom d, IbmSumArgs A);
__global__ void k_compute_C_S(Dom d, const double *xc, const double *yc, const double *geo, const int *ngeo,
                              double shift, double denom, double extra, double *CS);

// learned warm start (pvof_cnn.cu)
__global__ void k_cnn_sumsq(Dom d, const double *a, const double *b, double *partials);
__global__ void k_cnn_residual(Dom d, BcMap mp, const double *rho, const double *rhs, const double *phi_prev,
                               double *r0);
__global__ void k_cnn_assemble(Dom d, const double *rho, const double *rhs, const double *phi_prev, const double *phi,
                               const DevScalars *sc, float *x, float *t);
__global__ void k_cnn_expand(Dom d, const float *y, double *e);
__global__ void k_cnn_galerkin(Dom d, BcMap mp, const double *rho, const double *e, const double *r0, const double *M,
                               double *partials);
__global__ void k_cnn_apply(Dom d, const double *e, const double *phi_prev, const DevScalars *sc, double *phi);

// constant-density Poisson solver (pvof_fft.cu)
__global__ void k_fft_forward(Dom d, int N, int logN, const double *rhs, double *hc, double inx);
__global__ void k_fft_tridiag(Dom d, int N, int NYp, const double *as_, const double *ap_, const double *an_,
                              const double *mw, double *hc, double *gam);
__global__ void k_fft_inverse(Dom d, int N, int logN, const double *hc, double *out);

__global__ void k_cg_biharmonic(BihArgs A);
__global__ void k_cg_velocity(VelArgs A);
__global__ void k_cg_pressure(PresArgs A);
__global__ void k_cg_pressure_fw(PresArgs A);
__global__ void k_cg_pressure_fwp(PresArgs A);

}  // namespace pvof
