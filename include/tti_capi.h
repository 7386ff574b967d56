/*
 * tti_capi.h -- C ABI of the B200 TTI/VTI pseudo-acoustic RTM library
 * (libtti_b200.so).
 *
 * Drop-in boundary for the hot path of MiniAppsForHPE's simulator2 /
 * kernels/ (paths below are relative to the reference's simulatorsForNvidia/
 * directory).  Two levels, as in the reference:
 *
 *   1. Per-kernel launchers with the reference launchers' argument lists and
 *      meaning: raw device pointers to FP32 volumes in the reference layout
 *      (x fastest, radius-4 halo on every axis, ldimx padded to 32 floats),
 *      inclusive interior index ranges, leading dimensions and a stream.
 *   2. A simulator object covering the simulator2SetUp call surface: grid
 *      and model setup, source, receivers, forward and adjoint time loops,
 *      device-resident snapshot save/restore, imaging condition, image
 *      readback.
 *
 * Error convention: where the reference aborts (CUDA_TRY / EMSL_VERIFY,
 * utils/cuda_utils.h:20-60, utils/emsl_error.h:21) every entry point here
 * returns a status code instead.  Nothing in the library aborts.
 *
 * Streams are passed as void* (a cudaStream_t); NULL is the legacy default
 * stream, which is what the reference simulator uses (kernel_base.h:32-40).
 * Only order 8 is supported, the order the reference simulator runs
 * (simulator2SetUp.h:103); other orders return TTI_EINVAL.
 */
#ifndef TTI_CAPI_H
#define TTI_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TTI_OK = 0,
    TTI_EINVAL = 1,   /* bad argument or unsupported configuration */
    TTI_ENOMEM = 2,   /* device or pinned-host allocation failed */
    TTI_ELAUNCH = 3,  /* kernel launch or CUDA runtime error */
    TTI_ETIMEOUT = 4, /* a bounded wait gave up */
    TTI_ESTATE = 5,   /* call out of order (e.g. read before any write) */
    TTI_ERANGE = 6,   /* a reduced-precision snapshot value saturated (results produced) */
    TTI_ETOOBIG = 7   /* request larger than a fixed-capacity buffer of the library */
};

typedef void* tti_stream_t;

/* Human-readable name of a status code (static string). */
const char* tti_status_string(int status);
/* Library version, e.g. "0.1.0" (static string). */
const char* tti_version(void);

/* ------------------------------------------------------------------------
 * 1. Per-kernel launchers.  Device pointers; the caller owns every volume
 *    (as cart_volume_regular_gpu owns them in the reference).
 * ---------------------------------------------------------------------- */

/* Six staggered first derivatives (shift -1/2) times buoyancy Model11.
 * Replaces kernel3_gpu_kernels::launch_fwd_kernel2_drv
 * (kernels/kernel_type2_fwd_drv.h:7-11). */
int tti_launch_fwd_kernel2_drv(const float* field1, const float* field2, const float* Model11, float* dfield1dx,
                               float* dfield1dy, float* dfield1dz, float* dfield2dx, float* dfield2dy,
                               float* dfield2dz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                               float invdx, float invdy, float invdz, int ldimx, int ldimy, int order,
                               tti_stream_t stream);

/* Forward TTI update field3/field4 += dt*rhs.  Replaces
 * launch_update_rho_fwd_main_loop_2_1 (kernels/kernel_type2_fwd.h:6-14).
 * The PML arguments must be NULL and pml_x/y/z false: the reference never
 * instantiates its PML path (kernel_type2_fwd.cu:641).  sponge_active is
 * accepted and ignored, as in the reference launcher (kernel_type2_fwd.cu:641
 * instantiates sponge_active=false). */
int tti_launch_update_rho_fwd_main_loop_2_1(
    float* field3, float* field4, const float* field1_dx, const float* field2_dx, const float* field1_dy,
    const float* field2_dy, const float* field1_dz, const float* field2_dz, const float* field1, const float* field2,
    const float* irho, const float* model1, const float* model2, const float* model3, const float* model4,
    const float* rx, const float* ry, const float* rz, float* pml_field1_xx, float* pml_field2_xx,
    float* pml_field1_yy, float* pml_field2_yy, float* pml_field1_zz, float* pml_field2_zz, const float* pml_ab_x,
    const float* pml_ab_y, const float* pml_ab_z, const float* sponge_ab_xx, const float* sponge_ab_yy,
    const float* sponge_ab_zz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx,
    int ldimy, float dt, double dx, double dy, double dz, int sponge_active, int order, int pml_x, int pml_y,
    int pml_z, tti_stream_t stream);

/* Adjoint derivatives and mixed-derivative rhs.  Replaces
 * adj_kernel3_derivatives::launch_adj_kernel2_drv
 * (kernels/kernel_type2_grad_snap.h:7-12).  Model volumes must be finite
 * and Model11 non-zero in the x/y/z halo (the temporaries are formed there).
 * Like the reference launcher it keeps no state: its scratch (16 bytes per
 * cell up to plane izend+4) is allocated and freed in stream order on
 * `stream` (cudaMallocAsync / cudaFreeAsync), so calls on different streams
 * never share memory and no call synchronizes the device; TTI_ENOMEM when
 * the allocation fails. */
int tti_launch_adj_kernel2_drv(float* dfield1dx, float* dfield2dx, float* dfield1dy, float* dfield2dy,
                               float* dfield1dz, float* dfield2dz, float* field3_rhs, float* field4_rhs,
                               const float* field1, const float* field2, const float* Model11, const float* model1,
                               const float* model2, const float* model3, const float* model4, const float* model5,
                               const float* model6, const float* model7, int ixbeg, int ixend, int iybeg,
                               int iyend, int izbeg, int izend, float invdxx, float invdyy, float invdzz,
                               float invdxy, float invdyz, float invdzx, int ldimx, int ldimy, int order, float dt,
                               float invdx, float invdy, float invdz, tti_stream_t stream);

/* Same computation and arguments as tti_launch_adj_kernel2_drv, with a
 * scratch that is never allocated: no counterpart in the reference.  For
 * callers that must not have the library allocate device memory (their own
 * pool holds HBM, their device pool is configured for their own use, or
 * they must know the footprint up front).  The scratch is a fixed array of
 * TTI_NOALLOC_SCRATCH_CELLS cells (16 MiB); a request with
 * ldimx * ldimy * (izend + 5) above that returns TTI_ETOOBIG.  The first
 * call on a device looks up the array's address and should come before any
 * stream capture; the address is kept for the process, so the entry point
 * does not survive cudaDeviceReset (or any new primary context) on that
 * device.  All calls on a device share the array: calls that overlap on the
 * GPU race and must be ordered by the caller. */
#define TTI_NOALLOC_SCRATCH_CELLS (1 << 20)
int tti_launch_adj_kernel2_drv_noalloc(float* dfield1dx, float* dfield2dx, float* dfield1dy, float* dfield2dy,
                                       float* dfield1dz, float* dfield2dz, float* field3_rhs, float* field4_rhs,
                                       const float* field1, const float* field2, const float* Model11,
                                       const float* model1, const float* model2, const float* model3,
                                       const float* model4, const float* model5, const float* model6,
                                       const float* model7, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                                       int izend, float invdxx, float invdyy, float invdzz, float invdxy,
                                       float invdyz, float invdzx, int ldimx, int ldimy, int order, float dt,
                                       float invdx, float invdy, float invdz, tti_stream_t stream);

/* Adjoint update.  Replaces kernel3_gpu_kernels::launch_update_adj_kernel_main_3
 * (kernels/kernel_type2_adj.h:8-14).  ab_* are float2 (A,B) sponge arrays
 * indexed by the global axis index; pml flags must be false. */
int tti_launch_update_adj_kernel_main_3(float* field3, float* field4, const float* field1_dx,
                                        const float* field2_dx, const float* field1_dy, const float* field2_dy,
                                        const float* field1_dz, const float* field2_dz, const float* field3_rhs,
                                        const float* field4_rhs, const float* ab_xx, const float* ab_yy,
                                        const float* ab_zz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                                        int izend, int ldimx, int ldimy, float dt, double dx, double dy, double dz,
                                        int pmlx, int pmly, int pmlz, int order, int sponge_active,
                                        tti_stream_t stream);

/* Density gradient grad -= irho*sum(adj*D+fwd + D-adj*fwd).  Replaces
 * launch_update_rho_gradient_rho (kernels/kernel_type2_grad.h:22-32).
 * grad is not offset (element 0 is the first interior point) and has its
 * own leading dimensions, as in the reference.  Its scratch is taken and
 * returned in stream order on `stream`, as in tti_launch_adj_kernel2_drv. */
int tti_launch_update_rho_gradient_rho(float* grad, const float* fwd_field1_dx, const float* fwd_field2_dx,
                                       const float* fwd_field1_dy, const float* fwd_field2_dy,
                                       const float* fwd_field1_dz, const float* fwd_field2_dz, const float* field1,
                                       const float* field2, const float* irho, const float* model1,
                                       const float* model2, const float* model3, const float* model4,
                                       const float* rx, const float* ry, const float* rz, int ixbeg, int ixend,
                                       int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy,
                                       int grad_ldimx, int grad_ldimy, double dx, double dy, double dz, int order,
                                       int simple_gradient, tti_stream_t stream);

/* Free-surface mirror of the six derivative volumes over whole XY planes
 * iz <= izbeg.  Replaces the kernel3_gpu_kernels::kernel_loop4_derivatives
 * launch of kernel_type2::kernel_loop4_derivative_impl
 * (kernels/kernel_type2_small.h:8-9, kernels/kernel_type2.cu:278-293). */
int tti_launch_kernel_loop4_derivatives(float* dfield1dx, float* dfield1dy, float* dfield1dz, float* dfield2dx,
                                        float* dfield2dy, float* dfield2dz, int xtot, int ytot, int izbeg,
                                        tti_stream_t stream);

/* Imaging condition grad_Vp += adj3*snap3 + adj4*snap4 over the interior.
 * snap/grad have no halo and leading dimensions (snx, sny); adj fields are
 * halo'd with (ldimx, ldimy).  Replaces the update_Vp_gradient launch of
 * kernel_type2::update_grad_loop_1_impl (kernels/kernel_type2_small.h:11-14,
 * kernels/kernel_type2.cu:305-330). */
int tti_launch_update_Vp_gradient(const float* snap_field3, const float* snap_field4, float* grad_Vp,
                                  const float* adj_field3, const float* adj_field4, int ixbeg, int ixend, int iybeg,
                                  int iyend, int izbeg, int izend, int snx, int sny, int ldimx, int ldimy,
                                  tti_stream_t stream);

/* grad_Vp *= -2*dt_xcorr/sqrt(model3).  kernels/kernel_type2_small.h:16-18. */
int tti_launch_finalize_Vp_gradient(const float* model3, float* grad_Vp, int ixbeg, int ixend, int iybeg,
                                    int iyend, int izbeg, int izend, int snx, int sny, int ldimx, int ldimy,
                                    float dt_xcorr, tti_stream_t stream);

/* p = A*p + B*dt*pdot over the interior; ab_* float2 (A,B) per global index.
 * Replaces kernel_base::kernel_loop2_inner (kernels/kernel_base.cu:82-140). */
int tti_launch_kernel_loop2(float* field1, float* field2, const float* field3, const float* field4, int ldimx,
                            int ldimy, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                            const float* ab_x, const float* ab_y, const float* ab_z, float dt, tti_stream_t stream);

/* Free surface on p,q: zero at izbeg, odd mirror above, whole XY planes.
 * Replaces kernel_base::kernel_loop4_inner (kernels/kernel_base.cu:142-187). */
int tti_launch_kernel_loop4(float* field1, float* field2, int ldimx, int ldimy, int izbeg, tti_stream_t stream);

/* Model parameters from per-cell (vp, eps, delta, vs, theta, phi) over n
 * cells (any layout, element-wise).  simulator2SetUp.cu:10-29 restated per
 * cell (the reference takes scalars). */
int tti_launch_init_cijs(const float* vp, const float* eps, const float* delta, const float* vs,
                         const float* theta, const float* phi, float* model1, float* model2, float* model3,
                         float* model4, float* model5, float* model6, float* model7, int64_t n,
                         tti_stream_t stream);

/* Pressure P = -(2p+q)/3 over n cells.  simulator2SetUp.cu:31-42,842-857. */
int tti_launch_compute_pressure(float* pressure, const float* field1, const float* field2, int64_t n,
                                tti_stream_t stream);

/* Type1 discretisation (constant density, centred second derivatives, no
 * first-derivative stage; kernels/kernel_type1_gpu_*.cu).  Same arguments
 * and meaning as the reference launchers; order 8 only; `simple` selects the
 * reference's unoptimised kernels there and is accepted and ignored here (one
 * implementation, following the optimised kernels: the reference's simple
 * forward kernel reads the yz diagonal for the |i| >= 2 zx taps,
 * kernels/helper_kernels_gpu.h:180-181, so the two reference kernels differ).
 * ABx/ABy/ABz are float2 (A,B) sponge arrays; ldimz is needed to check the
 * z halo. */

/* Replaces fwd_main_loop_2_1_inner_gpu::launch (kernels/kernel_type1_gpu_fwd.h:6-9).
 * calc_snap = 0: field3/4 += dt*rhs (use_sponge = 0) or A*f + B*dt*rhs;
 * calc_snap = 1: rhs itself into halo-free field3/4 with ldimx_out/ldimy_out. */
int tti_launch_type1_fwd(float* field3, float* field4, const float* field1, const float* field2, const float* model1,
                         const float* model2, const float* model3, const float* model4, const float* model5,
                         const float* model6, const float* model7, const float* ABx, const float* ABy,
                         const float* ABz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                         int ldimx_in, int ldimy_in, int ldimz_in, int ldimx_out, int ldimy_out, int ldimz_out,
                         float dt, double dx, double dy, double dz, int order, tti_stream_t stream, int calc_snap,
                         int use_sponge, int simple);

/* Replaces adj_main_loop_2_inner_gpu::launch (kernels/kernel_type1_gpu_adj.h:6-9):
 * field3/4 += dt * D(M^T (field1, field2)) (or the sponge form).  Its
 * four-float scratch over the halo'd range is taken and returned in stream
 * order on `stream`, as in tti_launch_adj_kernel2_drv. */
int tti_launch_type1_adj(float* field3, float* field4, const float* field1, const float* field2, const float* model1,
                         const float* model2, const float* model3, const float* model4, const float* model5,
                         const float* model6, const float* model7, const float* ABx, const float* ABy,
                         const float* ABz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                         int ldimx, int ldimy, int ldimz, float dt, double dx, double dy, double dz, int order,
                         tti_stream_t stream, int use_sponge, int simple);

/* Replaces launch_update_grad_loop_kernel (kernels/kernel_type1_gpu_grad.h:4-7):
 * grad += adj_x*snap_x + adj_z*snap_z; snapshots and gradient halo-free with
 * leading dimensions snap_ldimx/snap_ldimy, adjoint volumes halo'd. */
int tti_launch_type1_update_grad(const float* snap_x, const float* snap_z, float* grad_Vp, const float* adj_x,
                                 const float* adj_z, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                                 int snap_ldimx, int snap_ldimy, int ldimx, int ldimy, tti_stream_t stream);

/* ------------------------------------------------------------------------
 * 2. Simulator object (simulator2SetUp call surface,
 *    simulator2/simulator2SetUp.h:25-35, execute at simulator2SetUp.cu:517-814).
 * ---------------------------------------------------------------------- */

typedef struct tti_sim tti_sim;

typedef struct {
    int nx, ny, nz;       /* interior grid (the reference's npoints+2*npml per axis) */
    double dx, dy, dz;    /* spacing (metres) */
    float dt;             /* time step (seconds) */
    int nt;               /* time steps (niter) */
    int xcorr_step;       /* snapshot / imaging cadence */
    int sponge_width;     /* absorbing cells on each side except a free-surface top; 0 = none */
    int free_surface;     /* 1: free surface at the top interior plane (reference behaviour) */
    int fused;            /* 1: fused step kernels; 0: the reference's kernel sequence */
    int save_snapshots;   /* 1: keep the forward snapshots on the device for the adjoint */
    int snap_precision;   /* snapshot storage: 0 FP32, 1 FP16, 2 BF16 (value * per-field power-of-two
                             scale; needs fused = 1 and nx a multiple of 8) */
    int checkpoint_every; /* 0: keep every snapshot of the shot.  K > 0 (a multiple of xcorr_step;
                             fused = 1, save_snapshots = 1): keep FP32 checkpoints of the forward
                             state every K steps and the snapshots of one K-step segment; the
                             adjoint recomputes each segment's snapshots from its checkpoint.
                             Results are identical to K = 0. */
    int use_graphs;       /* 1: each time loop (or checkpoint segment) is captured into a CUDA graph
                             and launched as one; the instantiated graph is reused across calls */
    int scheme;           /* 0: staggered variable-density operator (kernel_type2, the simulator's
                             own); 1: centred constant-density operator (kernel_type1 launchers;
                             Vp image only, grad_rho stays zero) */
    int wave_precision;   /* 0: FP32 wavefields.  1 FP16 / 2 BF16 (fused = 1): p and q leave every
                             step rounded to that format of value * a per-field power-of-two scale
                             (from the previous step's largest |p|, |q|) and are read back exactly;
                             stencils, pdot/qdot and the time update stay FP32.  The rounded
                             values are held in the FP32 arrays (the stencil kernels are
                             instruction-bound, not byte-bound), so this is the numerics of
                             FP16/BF16 wavefield storage without its memory saving. */
} tti_sim_config;

int tti_sim_create(const tti_sim_config* cfg, tti_sim** out);

/* Device bytes a simulator with this configuration allocates at creation
 * (receiver buffers, nt*nrec*8 bytes + nrec*8, come on top at
 * tti_sim_set_receivers).  Used for admission by HBM footprint. */
int tti_sim_footprint_bytes(const tti_sim_config* cfg, int64_t* bytes);
int tti_sim_destroy(tti_sim* sim);

/* Model from host arrays over the interior (nx*ny*nz, x fastest): vp, eps,
 * delta, vs (m/s), theta, phi (radians), rho.  Halos are filled by edge
 * extension.  Any pointer may be NULL for its default (eps=delta=vs=theta=phi=0,
 * rho=1). */
int tti_sim_set_model(tti_sim* sim, const float* vp, const float* eps, const float* delta, const float* vs,
                      const float* theta, const float* phi, const float* rho);

/* Point source at interior cell (ix,iy,iz): pdot,qdot += w[n]*dt each step. */
int tti_sim_set_source(tti_sim* sim, int ix, int iy, int iz, const float* wavelet_host, int nt);

/* Receivers at interior cells (3*nrec ints: ix,iy,iz per receiver, distinct).
 * They record P = -(2p+q)/3 every step. */
int tti_sim_set_receivers(tti_sim* sim, int nrec, const int* ixyz_host);

/* Forward time loop (nt steps).  traces: nt*nrec floats, host memory if
 * traces_on_device is 0 else device memory; may be NULL. */
int tti_sim_forward(tti_sim* sim, float* traces, int traces_on_device);

/* Adjoint time loop seeded with residual traces (nt*nrec, same placement
 * rule), imaging condition at every snapshot step (Vp and rho gradients). */
int tti_sim_adjoint(tti_sim* sim, const float* residual, int residual_on_device);

/* Adjoint loop whose residual is formed on the device from the synthetic
 * traces of the last forward run minus these observed traces (nt*nrec). */
int tti_sim_adjoint_observed(tti_sim* sim, const float* observed, int observed_on_device);

/* Failure-detection self-check (no reference counterpart; the reference
 * aborts instead).  Every wait inside the fused kernels is bounded: a wait
 * that runs out records a timeout that the simulator returns as
 * TTI_ETIMEOUT, and the kernel returns, leaving the context usable.  This
 * runs that path on a shared-memory barrier that nothing completes, with a
 * limit of `seconds` (0 < seconds <= 10) of SM clock cycles; it returns
 * TTI_ETIMEOUT when the wait gave up and reported as it should. */
int tti_selfcheck_bounded_wait(double seconds, tti_stream_t stream);

/* z-chunk autotuner.  The fused kernels run one CTA per SM on TX x TY
 * column tiles (TX = 32, TY = 16) marching along z; the grid's planes are
 * split among CTAs in tile-major order, bz consecutive planes per CTA (one
 * or more column segments, each paying a pipeline fill of 14 planes), so bz
 * sets how many CTAs a step launches against the fill overhead.
 * tti_sim_autotune times every candidate split (whole-column chunks
 * ceil(nz/n), equal shares for 1..8 CTAs per SM of at least 8 planes, and,
 * on grids with fewer tile columns than SMs, top/bottom splits as for
 * tti_tune_set_split around the balance point of the tops) of the fused
 * forward, adjoint and (with a snapshot store) imaging kernels on this
 * simulator's volumes, reps launches each, times the three fastest (and the
 * fastest top/bottom split, if within 3 %) again with more launches and
 * records the fastest (a top/bottom split within 1 % of it is taken
 * instead: same speed, about half the DRAM traffic) for this
 * grid on the current device; later launches on any simulator of the same
 * grid use it.  Needs fused = 1 and a model.  Wavefield and image contents
 * afterwards are unspecified (forward and adjoint start from zero).  The
 * split changes only the launch shape: results do not depend on bz. */
typedef struct {
    int bz[3];         /* chosen bz: forward, adjoint, imaging (0: not tuned); with scheme = 1
                          the centred forward and adjoint kernels, imaging not tuned */
    int ztop[3];       /* chosen top/bottom split (0: plain tile-major bz) */
    float ms[3];       /* per-launch time at the chosen bz */
    float model_ms[3]; /* per-launch time at the wave-count model's bz */
    int ncand;         /* candidates tried per kernel */
} tti_tune_report;
int tti_sim_autotune(tti_sim* sim, int reps, tti_tune_report* out);

/* Record (bz > 0) or clear (bz = 0) the planes per CTA used for kernel kind
 * (0 forward, 1 adjoint, 2 imaging of the staggered scheme; 3 forward,
 * 4 adjoint of the centred scheme) on an nx*ny*nz grid, current device;
 * tti_tune_get returns the bz in effect (recorded or modelled). */
int tti_tune_set(int nx, int ny, int nz, int kind, int bz);
int tti_tune_get(int nx, int ny, int nz, int kind);
/* The same with a top/bottom split: ztop > 0 gives each of the grid's T
 * tile columns a CTA for its top ztop planes and lets further CTAs share
 * the columns' bottoms (planes ztop .. nz-1), bz planes each; ztop = 0 is
 * the plain tile-major split of tti_tune_set. */
int tti_tune_set_split(int nx, int ny, int nz, int kind, int bz, int ztop);
int tti_tune_get_split(int nx, int ny, int nz, int kind, int* bz, int* ztop);

/* Step-level calls for a caller that keeps its own time loop (the loop body
 * of simulator2SetUp::execute, simulator2/simulator2SetUp.cu:517-814): the
 * kernels of tti_sim_forward / tti_sim_adjoint, one time step per call,
 * enqueued on the simulator's stream without synchronising.  Needs
 * checkpoint_every = 0 and use_graphs = 0.  Calls out of order return
 * TTI_ESTATE.
 *   tti_sim_forward_begin: zero the wavefields (fused: and the step-0 p/q
 *     update); then tti_sim_forward_step for n = 0 .. nt-1 in order: receiver
 *     sample, the step, the snapshot at n % xcorr_step == 0;
 *     tti_sim_get_traces reads the traces back (synchronises).
 *   tti_sim_adjoint_begin: zero the adjoint wavefields and images and take
 *     the residual traces (nt*nrec, as tti_sim_adjoint; NULL = zero); then
 *     tti_sim_adjoint_step for n = nt-1 .. 0 in order (residual injection and
 *     the adjoint step), each snapshot step n optionally followed by
 *     tti_sim_image_step(n) (Vp and rho images from the stored snapshot);
 *     tti_sim_adjoint_finish after step 0 finalises the Vp image,
 *     synchronises and returns the bounded-wait status.
 *   tti_sim_sync: synchronise the stream and return that status. */
int tti_sim_forward_begin(tti_sim* sim);
int tti_sim_forward_step(tti_sim* sim, int n);
int tti_sim_get_traces(tti_sim* sim, float* traces, int on_device);
int tti_sim_adjoint_begin(tti_sim* sim, const float* residual, int residual_on_device);
int tti_sim_adjoint_step(tti_sim* sim, int n);
int tti_sim_image_step(tti_sim* sim, int n);
int tti_sim_adjoint_finish(tti_sim* sim);
int tti_sim_sync(tti_sim* sim);

/* Image readback: Vp gradient (finalised, -2*dt*xcorr/vp) and rho gradient,
 * nx*ny*nz each, host or device memory. */
int tti_sim_get_image(tti_sim* sim, float* grad_vp, float* grad_rho, int on_device);

/* Gradient of the receiver misfit of the last adjoint run with respect to
 * each source wavelet sample: dt*(adjoint p + q) at the source cell, nt
 * floats into host memory.  Together with tti_sim_forward this gives the
 * forward/adjoint pair a dot-product test can check. */
int tti_sim_source_gradient(tti_sim* sim, float* host_out);

/* Device pointer of an internal volume for inspection: which = 0..3 for
 * field1..field4 (p, q, pdot, qdot), 4..11 for irho, model1..model4, rx, ry, rz. */
int tti_sim_volume(tti_sim* sim, int which, float** dev_ptr);

/* Copy one internal volume (same numbering as tti_sim_volume) to host
 * memory: ldimx*ldimy*ldimz floats. */
int tti_sim_read_volume(tti_sim* sim, int which, float* host_dst);

/* Layout of the simulator's volumes: ldimx, ldimy, ldimz. */
int tti_sim_layout(tti_sim* sim, int* ldimx, int* ldimy, int* ldimz);

/* Per-launch timing of the step kernels with CUDA events on the simulator's
 * stream (enable resets the totals).  tti_sim_kernel_times fills ms[3] and
 * launches[3] for: 0 forward step kernel, 1 adjoint step kernel, 2 imaging. */
int tti_sim_set_profiling(tti_sim* sim, int enable);
int tti_sim_kernel_times(tti_sim* sim, double* ms, int64_t* launches);

/* Kernel launches issued by the last forward/adjoint call. */
int64_t tti_sim_launch_count(tti_sim* sim);

/* Stream the simulator runs on (a cudaStream_t). */
tti_stream_t tti_sim_stream(tti_sim* sim);

/* ------------------------------------------------------------------------
 * 3. Device-resident snapshot store with the rtm_snap call sequence
 *    (snap_helpers/rtm_snap.h:19-41): LIFO, written on the forward pass,
 *    read back in reverse on the adjoint pass.  Each snapshot holds nvol
 *    volumes of the given element counts.
 * ---------------------------------------------------------------------- */
typedef struct tti_snap_store tti_snap_store;

int tti_snap_create(int nvol, const int64_t* nelem, int capacity, tti_snap_store** out);
/* Store with a host tier: device_capacity slots in HBM, then host_capacity
 * slots in pinned host memory (the reference's host-RAM buffers,
 * snap_helpers/file_snap_orig.cpp:221-352); the same call sequence moves
 * snapshots to and from either tier on the store's copy stream. */
int tti_snap_create_tiered(int nvol, const int64_t* nelem, int device_capacity, int host_capacity,
                           tti_snap_store** out);
int tti_snap_destroy(tti_snap_store* s);
/* Waits for the previous write to have drained (rtm_snap lock_for_write). */
int tti_snap_lock_for_write(tti_snap_store* s);
/* Copies the nvol device volumes into the next slot, ordered after work
 * already queued on stream (rtm_snap start_write). */
int tti_snap_start_write(tti_snap_store* s, float* const* vols, tti_stream_t stream);
/* Starts copying the most recent unread slot into the nvol device volumes
 * (rtm_snap start_read); TTI_ESTATE when the store is empty. */
int tti_snap_start_read(tti_snap_store* s, float* const* vols, tti_stream_t stream);
/* Orders stream after the pending read (rtm_snap finish_read). */
int tti_snap_finish_read(tti_snap_store* s, tti_stream_t stream);
int tti_snap_count(tti_snap_store* s);

/* ------------------------------------------------------------------------
 * 4. Shot server: continuous batching of RTM shots on one device.  No
 *    counterpart in the reference (one shot per run there).
 *
 *    Shots of any grid size are queued, admitted first-fit in arrival order
 *    while the number of resident shots is below max_active and their device
 *    footprint (tti_sim_footprint_bytes plus receiver and set-up buffers)
 *    fits the HBM budget, and then stay resident (wavefields, snapshot store,
 *    checkpoints) until their image is read back.  A shot that would not fit
 *    the budget alone gets checkpointed recomputation.  The scheduler runs in
 *    rounds: each round advances every resident shot by a number of fused
 *    steps sized to take about round_ms of device time, all shots in
 *    parallel branches of one launch (one captured CUDA graph when
 *    use_graphs = 1); the next round is prepared while the current one runs,
 *    and shots admitted in the meantime join it.  Each shot computes exactly
 *    what tti_sim_forward + tti_sim_adjoint_observed compute for it alone.
 * ---------------------------------------------------------------------- */
typedef struct tti_server tti_server;

typedef struct {
    int max_active;      /* shots resident at once (>= 1) */
    int64_t hbm_budget;  /* device bytes for shots; 0 = free memory at creation minus 2 GiB */
    float round_ms;      /* target device time of one round (> 0) */
    int use_graphs;      /* 1: one captured graph launch per round */
    int autotune;        /* 1: tune the z-chunk of each new grid size before its first shot */
    int snap_precision;  /* snapshot store of every shot: 0 FP32, 1 FP16, 2 BF16 */
    int scheme;          /* operator of every shot: 0 staggered variable-density, 1 centred
                            constant-density (as tti_sim_config.scheme) */
} tti_server_config;

/* One shot.  Host arrays only; the server reads and writes them while the
 * shot is queued or resident, so they must stay valid until its result has
 * been taken with tti_server_wait. */
typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
    float dt;
    int nt, xcorr_step, sponge_width, free_surface;
    const float *vp, *eps, *delta, *vs, *theta, *phi, *rho; /* nx*ny*nz; NULL = default */
    int src_ix, src_iy, src_iz;
    const float* wavelet;  /* nt */
    int nrec;
    const int* rec_ixyz;   /* 3*nrec */
    const float* observed; /* nt*nrec observed traces; NULL = zero (residual = synthetic) */
    float* image_vp;       /* out, nx*ny*nz, may be NULL */
    float* image_rho;      /* out, nx*ny*nz, may be NULL */
    float* traces;         /* out, nt*nrec synthetic traces, may be NULL */
} tti_shot_request;

typedef struct {
    int status;                       /* TTI_OK or the failing call's status */
    double t_submit, t_admit, t_done; /* seconds on the server's clock (tti_server_now) */
    int64_t footprint;                /* device bytes reserved for the shot */
    int checkpoint_every;             /* 0 or the segment length chosen at admission */
    int64_t units;                    /* fused steps run (forward, recomputed, adjoint) */
    int64_t launches;                 /* kernel launches of the shot */
} tti_shot_result;

typedef struct {
    int64_t rounds;               /* batched launches */
    int64_t graph_updates;        /* rounds whose graph was updated in place */
    int64_t graph_instantiations;
    int max_resident;             /* most shots resident at once */
    double busy_ms;               /* device time of all rounds */
    double gap_ms;                /* device idle between a round and the one issued behind it
                                     (the host was late with the next round) */
    double build_ms;              /* host time spent capturing, updating and launching rounds */
    double setup_ms;              /* host time spent admitting shots (allocation, model upload,
                                     autotuning a new grid) */
    int max_batched;              /* most shots advanced in one round */
    double setup_alloc_ms;        /* of setup_ms: creating the shots' simulators (device allocation) */
    double setup_model_ms;        /* of setup_ms: model, source, receiver and observed-trace upload */
    double setup_tune_ms;         /* of setup_ms: autotuning new grid sizes */
} tti_server_stats;

/* Run-level call: one whole shot from host arrays, synchronously, on a
 * simulator created and destroyed for it (forward with receivers, adjoint
 * driven by observed - synthetic traces, or by the synthetic traces when
 * observed is NULL, images into image_vp / image_rho).  opts (NULL =
 * defaults) contributes only fused, snap_precision, checkpoint_every,
 * use_graphs, scheme and wave_precision; the physical set-up comes from
 * the request. */
int tti_rtm_shot(const tti_shot_request* req, const tti_sim_config* opts);

int tti_server_create(const tti_server_config* cfg, tti_server** out);
int tti_server_submit(tti_server* srv, const tti_shot_request* req, int64_t* ticket);
/* Waits up to timeout_s seconds (< 0: no limit) for the shot; TTI_ETIMEOUT
 * if it is not done by then.  A result is handed out once. */
int tti_server_wait(tti_server* srv, int64_t ticket, double timeout_s, tti_shot_result* out);
int tti_server_stats_get(tti_server* srv, tti_server_stats* out);
double tti_server_now(tti_server* srv);
/* Runs every submitted shot to completion, then releases the server. */
int tti_server_destroy(tti_server* srv);

/* ------------------------------------------------------------------------
 * 5. Elastic step kernels of the reference's simulator3 (its eTTI proxy),
 * with the reference's stand-in constants (first-derivative and
 * interpolation tables {1.01, 2.01, 3.01, 4.01}, inverse spacings 1.01 and
 * 2.01 or 2.02 in x and y, zprime[iz] in z) and arithmetic.  Volumes are
 * FP32, x fastest, radius-4 halo on every axis, interior [4, 4+n-1] per
 * axis, idx = (iz*ldimy + iy)*ldimx + ix, ldimx >= nx + 8, ldimy >= ny + 8,
 * and the z allocation holds nz + 8 planes; zprime is indexed by the halo'd
 * z.  The reference launches need nx a multiple of 32 and ny of 16 (its
 * blocks check no bounds); these take any size and write interior cells
 * only.  stream 0 is the default stream. */

/* Replaces vgPlainLoop (simulator3/simulator3SetUp.cu:1364-1386): the six
 * strain volumes d4..d9 from the velocities f1, f2, f3. */
int tti_e3_launch_vgplain(const float* f1, const float* f2, const float* f3, float* d4, float* d5, float* d6,
                          float* d7, float* d8, float* d9, const float* zprime, int nx, int ny, int nz, int ldimx,
                          int ldimy, tti_stream_t stream);

/* Replaces sPlainLoop (simulator3/simulator3SetUp.cu:1127-1216): the six
 * z-mixed precomputes into f10_21[0..11] (the reference's f10 .. f21, in its
 * 64-plane z blocks, whose first planes it weighs differently), then the
 * stress update f4..f9 += C:strain with M[0..20] = M1..M21 and the strains
 * f1_1, f1_2, f1_3, f2_2, f2_3, f3_3 (the simulator passes d4 .. d9). */
int tti_e3_launch_splain(float* f4, float* f5, float* f6, float* f7, float* f8, float* f9, const float* const* M,
                         const float* f1_1, const float* f1_2, const float* f1_3, const float* f2_2,
                         const float* f2_3, const float* f3_3, float* const* f10_21, int nx, int ny, int nz,
                         int ldimx, int ldimy, tti_stream_t stream);

/* Replaces vPlainLoop (simulator3/simulator3SetUp.cu:1105-1125): the
 * velocity update f1..f3 += 2*M22 * div(stress f4..f9). */
int tti_e3_launch_vplain(float* f1, float* f2, float* f3, const float* f4, const float* f5, const float* f6,
                         const float* f7, const float* f8, const float* f9, const float* M22, const float* zprime,
                         int nx, int ny, int nz, int ldimx, int ldimy, tti_stream_t stream);

/* Replaces mirror_s / mirror_v (simulator3/simulator3SetUp.cu:1425-1492):
 * on nfields (1..6) volumes, plane izbeg set to zero and planes 0..izbeg-1
 * to the negated mirror 2*izbeg - iz, whole planes (halos included);
 * ldimz (the planes allocated) bounds the mirror: 2*izbeg < ldimz. */
int tti_e3_launch_mirror(float* const* fields, int nfields, int ldimx, int ldimy, int ldimz, int izbeg,
                         tti_stream_t stream);

/* Replaces update_gv / update_g_v (simulator3/simulator3SetUp.cu:1494-1538):
 * the velocity image g1 += a_v1 * snap_v1 + a_v3 * snap_v3 over the nx*ny*nz
 * interior, g1 and the snapshots halo-free with leading dimensions g_ldimx,
 * g_ldimy, the adjoint velocities halo'd (ldimx, ldimy).  The density image
 * of the same schedule (update_g_r_impl, :2091-2128) is the TTI density
 * gradient with the elastic volumes in its argument slots:
 * tti_launch_update_rho_gradient_rho. */
int tti_e3_launch_update_gv(float* g1, const float* snap_v1, const float* snap_v3, const float* a_v1,
                            const float* a_v3, int nx, int ny, int nz, int ldimx, int ldimy, int g_ldimx, int g_ldimy,
                            tti_stream_t stream);

/* Replaces compute_p_kernel (simulator3/simulator3SetUp.cu:275-289) over n
 * cells: p = -(2 f4 + 3 f5 + 4 f6 + 5 f7 + 6 f8 + 7 f9) / 27. */
int tti_e3_launch_compute_p(float* p, const float* f4, const float* f5, const float* f6, const float* f7,
                            const float* f8, const float* f9, int64_t n, tti_stream_t stream);

/* Replaces init_cijs_kernel (simulator3/simulator3SetUp.cu:229-273): the
 * stand-in model M[0..21] = M1..M22, the strains d4_9[0..5] = d4..d9 and
 * zprime, from cos/sin of the halo'd cell indices, over the interior x range
 * and every y and z of the allocation (ldimz planes), as the reference's
 * launch covers them. */
int tti_e3_launch_init_model(float* const* M22, float* const* d4_9, float* zprime, int nx, int ldimx, int ldimy,
                             int ldimz, tti_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* TTI_CAPI_H */
