/*
 * symphas_b200.h -- C ABI of the B200 explicit finite-difference engine.
 *
 * This is the boundary between a host caller (the C++ MODEL/EVOLUTION front
 * end in include/symphas_b200/, the Python package, or any FFI) and the
 * sm_100a kernels.  Plain C types only; every call returns an int status
 * (SP_OK = 0) and never throws; sp_last_error() gives the message of the last
 * failure on a handle.
 *
 * What each entry point replaces in SymPhas (paths inside the SymPhas tree):
 *
 *   sp_create    Model<D,Sp,S...>(coeff, ncoeff, params) with
 *                SolverFT<Stencil2d2h<L,G,B>|Stencil3d2h<L,G,B>>:
 *                systems and dframe construction (sol/inc/model.h:100-128),
 *                SolverFT::make_solver (examples/solvers/solverft.h:121-161),
 *                StencilBase{2,3}d2h divh powers (sol/inc/stencilincludes.h:95-135)
 *   sp_upload    writing the interior of system<i>().values
 *                (sol/inc/solversystem.h:51-59) followed by update(t), the
 *                halo refresh (datatypes/inc/boundaryupdate.h:154-356)
 *   sp_step      n iterations of model_iteration: equation() then step(dt)
 *                then update(t) (modules-models.h:435-467;
 *                examples/solvers/solverft.h:46-50, :90-103)
 *   sp_download  reading the interior of system<i>().values / get_field<i>()
 *   sp_reduce    the density and energy collectors evaluated at save points
 *                (dataprocesses/datadensity.h, dataprocesses/dataenergy.h)
 *   sp_destroy   ~Model
 *
 * Threading: a handle is used by one host thread at a time; all its work runs
 * in order on one CUDA stream (its own, or the one given by sp_set_stream).
 * Ownership: the handle owns its device buffers; the caller owns host buffers.
 */
#ifndef SYMPHAS_B200_H
#define SYMPHAS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SP_OK 0
#define SP_EINVAL 1      /* bad argument or unsupported combination */
#define SP_ECUDA 2       /* a CUDA runtime call failed */
#define SP_ENOMEM 3      /* device allocation failed */
#define SP_ETIMEOUT 4    /* a bounded device wait gave up (error flag set by a kernel) */
#define SP_ENONFINITE 5  /* a reduction saw NaN or Inf */

/* dtype of the fields on the device */
#define SP_F32 0
#define SP_F64 1

/* boundary kind of one side (order LEFT RIGHT TOP BOTTOM FRONT BACK, i.e.
 * x-, x+, y-, y+, z-, z+ as in Side, lib/inc/definitions.h:588) */
#define SP_PERIODIC 0
#define SP_DIRICHLET 1 /* BoundaryType::DEFAULT with BoundaryTag::CONSTANT */

/* built-in models (each lowered at build time into fused kernels) */
#define SP_MODEL_A 0      /* MA:  dpsi = lap(psi) + (c1 - c2 psi^2) psi                */
#define SP_MODEL_B 1      /* MB:  dpsi = -bilap(psi) - lap((c1 - c2 psi^2) psi)        */
#define SP_MODEL_C 2      /* two fields psi, eta; gamma = c1:
                             dpsi = lap(-psi + psi^3 + 2 gamma psi eta^2 - lap psi)
                             deta = eta - eta^3 - 2 gamma psi^2 eta + lap eta          */
#define SP_MODEL_AMK 3    /* dpsi = M (kappa lap psi - psi^3 + psi), M = c1, kappa = c2 */
#define SP_MODEL_BMK 4    /* dpsi = M lap(psi^3 - psi - kappa lap psi)                  */
#define SP_OP_LAP 10      /* dframe = lap(psi)       (single-operator models used to   */
#define SP_OP_BILAP 11    /* dframe = bilap(psi)      check every stencil point set)    */
#define SP_OP_GRADLAP 12  /* dframe = x component of gradlap(psi)                       */
#define SP_OP_LAPCUBE 13  /* dframe = lap(psi^3)                                        */

/* evaluation form */
#define SP_FORM_EXACT 1 /* the printed scheme of SymPhas, term by term, no FMA
                           contraction: bit-identical to the CPU solver in FP64 */
#define SP_FORM_FUSED 0 /* algebraically equal fused form (bilap = lap o lap,
                           derivatives of a sum merged, staged in shared memory) */

typedef struct sp_desc {
  int dim;              /* 2 or 3 */
  int n[3];             /* interior extents x, y, z (z ignored when dim == 2) */
  int dtype;            /* SP_F32 or SP_F64 */
  int model;            /* SP_MODEL_* or SP_OP_* */
  int form;             /* SP_FORM_EXACT or SP_FORM_FUSED */
  int lap_pts;          /* Stencil2d2h<L,G,B> / Stencil3d2h<L,G,B> point counts */
  int gradlap_pts;
  int bilap_pts;
  int boundary[6];      /* SP_PERIODIC or SP_DIRICHLET per side */
  double boundary_value[6];
  double h;             /* uniform grid spacing */
  double dt;            /* forward-Euler time step */
  double coeff[8];      /* c(1)..c(8); unused entries should be 1 (c(i) default) */
  int ncoeff;
  int batch;            /* number of identical independent instances (>= 1) */
  int accuracy;         /* order of accuracy of the stencils: 2 (or 0):
                           Stencil2d2h / Stencil3d2h; 4: Stencil2d4h
                           (sol/inc/stencilh4.h; 2D only) */
} sp_desc;

typedef struct sp_handle sp_handle;

/* Create a handle: validates the description, allocates the device fields
 * (interior + halo, ping-pong) and builds the TMA descriptors. */
int sp_create(const sp_desc* desc, sp_handle** out);

/* ---- ensembles of independent 2D systems --------------------------------
 * One member of an ensemble: its own interior extents (x, y; n[2] unused),
 * model (SP_MODEL_*), time step and coefficients c(1)..c(8).  SymPhas runs
 * such a sweep as one Model object per member, stepped one after another by
 * find_solution (modules-io.h:747-753); here every member advances in the same
 * persistent kernel launch, which takes (member, tile) work items from one
 * queue, so small and large members share the GPU without a launch each. */
typedef struct sp_member {
  int n[3];
  int model;
  double dt;
  double coeff[8];
} sp_member;

/* model id reported for an ensemble that mixes SP_MODEL_AMK and SP_MODEL_BMK
 * members (one kernel holding both right-hand sides) */
#define SP_ENSEMBLE_AMK_BMK 5

/* Create a handle over `count` members.  `desc` gives what they share: dim
 * (must be 2), dtype, form, stencil point counts, boundaries and h; its n,
 * model, dt, coeff and batch are ignored.  The members either all have one
 * model, or mix SP_MODEL_AMK and SP_MODEL_BMK.  Instance i of the handle is
 * member i: sp_upload, sp_download, sp_fill_uniform, sp_reduce and
 * sp_field_geometry take its own extents; sp_step advances every member by
 * its own dt; sp_set_dt is rejected. */
int sp_create_ensemble(const sp_desc* desc, const sp_member* members, int count,
                       sp_handle** out);

/* Copy `bytes` of interior values (x-fastest, dtype of the handle) of field
 * `field` of instance `inst` from host memory, then refresh its halo. */
int sp_upload(sp_handle* h, int inst, int field, const void* host, size_t bytes);
/* Same from device memory (bytes in the same compact interior layout). */
int sp_upload_device(sp_handle* h, int inst, int field, const void* dev, size_t bytes);
/* Fill field `field` of instance `inst` with the seeded SplitMix64 stream
 * value(i) = lo + (hi - lo) * u53(seed, i), bit-identical to the oracle. */
int sp_fill_uniform(sp_handle* h, int inst, int field, uint64_t seed, double lo, double hi);

/* Advance every instance by `nsteps` forward-Euler iterations. */
int sp_step(sp_handle* h, int nsteps);

/* Keep the mass of field 0 of every instance at its present value: from now
 * on, after every `every` steps, sp_step reduces each instance's mass in FP64
 * and shifts the field uniformly (interior and periodic halo) so the mass
 * returns to the value it had at this call; every = 0 turns it off.  For
 * conserved fields (models B, BMK, field psi of C) in FP32, whose stored
 * values round at every step; all queued on the handle's stream, no host
 * wait.  Needs periodic boundaries on every axis.  No counterpart in SymPhas,
 * whose FP64 steps need none. */
int sp_conserve_mass(sp_handle* h, int every);

/* Advance every instance by `nsteps` (>= 1) iterations; the last one also sums
 * field 0 of each instance in FP64 inside the step kernel (warp shuffles) and
 * writes the `batch` sums to `mass`.  Waits for the result. */
int sp_step_mass(sp_handle* h, int nsteps, double* mass);

/* Evaluate the right-hand side (dframe) of the current state once, without
 * stepping, and copy field `field` of instance `inst` to host memory. */
int sp_eval_rhs(sp_handle* h, int inst, int field, void* host, size_t bytes);

/* Copy the interior of field `field` of instance `inst` to host memory and
 * wait for the copy. */
int sp_download(sp_handle* h, int inst, int field, void* host, size_t bytes);
/* Same into device memory (compact interior layout), stream-ordered. */
int sp_download_device(sp_handle* h, int inst, int field, void* dev, size_t bytes);
/* One field of every instance at once, to or from a dense device array
 * [instance][interior, x fastest] (`bytes` = batch x sites x element size):
 * one copy kernel, and after an upload one halo refresh for the whole batch
 * (periodic images, Dirichlet constants), where sp_upload_device per instance
 * takes a copy and two halo launches each.  The instances must share their
 * extents (a batch of one model, or an ensemble of equal members).  No
 * counterpart in SymPhas (one host copy per system's `values`). */
int sp_upload_batch_device(sp_handle* h, int field, const void* dev, size_t bytes);
int sp_download_batch_device(sp_handle* h, int field, void* dev, size_t bytes);

/* FP64 reductions over the interior of field `field` of instance `inst`:
 * mass = sum of values (SymPhas's Density collector,
 * dataprocesses/datadensity.h:11-19; its Energy collector is that sum over
 * the number of sites, dataprocesses/dataenergy.h:11-19), energy = h^D * sum
 * of a Landau free-energy density (forward-difference gradients; no SymPhas
 * counterpart):
 *   A, B:      -c1 v^2 / 2 + c2 v^4 / 4 + |grad v|^2 / 2
 *   AMK, BMK:  -v^2 / 2 + v^4 / 4 + c2 |grad v|^2 / 2
 *   C:         the same for psi and eta with unit coefficients, + c1 psi^2 eta^2
 * The mass is not scaled by h^D.  Waits for the result; SP_ENONFINITE when a
 * sum is NaN or infinite. */
int sp_reduce(sp_handle* h, int inst, int field, double* mass, double* energy);

/* Time every tile shape built for this kernel on this GPU (`reps` launches
 * each, per step; the fields are not changed: one-step kernels evaluate the
 * right-hand side, temporally blocked ones write their steps into the buffer
 * that is not current) and keep the fastest, which fixes the temporal-block
 * depth too; later sp_create calls with the same kernel and size in the same
 * process start with it.  No counterpart in SymPhas. */
int sp_autotune(sp_handle* h, int reps);
/* Steps one launch of the chosen kernel advances (its temporal-block depth):
 * 1 for the one-step kernels; k > 1 for a temporally blocked 2D kernel, which
 * sp_step then launches once per k steps (and once with fewer steps for a
 * remainder).  No counterpart in SymPhas (SolverFT takes one step per call of
 * Solver::step, examples/solvers/solverft.h:46-103). */
int sp_steps_per_launch(const sp_handle* h, int* kt);
/* The chosen kernel shape: {tile x, tile y, rows per thread, TMA stages in
 * flight, variant index, number of variants, threads per CTA, z planes per
 * CTA (3D) or persistent CTAs (2D)}. */
int sp_kernel_info(const sp_handle* h, int info[8]);

/* Change the time step of further sp_step calls (SolverFT's dt, set by
 * Model::step at sol/inc/model.h:932-936). */
int sp_set_dt(sp_handle* h, double dt);

/* Run all further work of the handle on `stream` (a cudaStream_t). */
int sp_set_stream(sp_handle* h, void* stream);
/* Wait until all queued work of the handle is done.  SP_ETIMEOUT when a
 * kernel gave up on a bounded wait since the last check; the handle's device
 * error flag is then cleared and its 2D work queue re-armed, so the handle
 * stays usable. */
int sp_synchronize(sp_handle* h);
/* Test hook for that failure path (no counterpart in SymPhas): queue on the
 * handle's stream one warp that waits `cycles` SM cycles (at most 2^31) on an
 * mbarrier nothing completes -- no copy is in flight -- then gives up as a
 * step kernel does and sets the device error flag; with `dirty_queue` it
 * first takes an item from the handle's 2D work queue without re-arming it.
 * The next synchronising call returns SP_ETIMEOUT. */
int sp_test_wait_timeout(sp_handle* h, long long cycles, int dirty_queue);
/* Number of fused-step kernel launches issued so far by this handle. */
long long sp_launch_count(const sp_handle* h);
/* Device pointer of the current interior origin of a field and its
 * padded geometry (pitch and halo in elements), for zero-copy callers. */
int sp_field_geometry(const sp_handle* h, int inst, int field, void** dev_origin,
                      long long* pitch, long long* plane, int halo[3]);

/* Structure factor of field `field` of instance `inst`, as SymPhas's SF
 * collector computes it (dataprocesses/datasf.h:137-245 with the radial
 * average of datatypes/inc/datalib.h:1120-1330): the interior, thresholded to
 * 1 where the value is positive and 0 elsewhere when `threshold` is nonzero
 * (SymPhas's choice) or taken as it is, is Fourier transformed (FP64), and
 * |F(k)|^2 / (number of sites) is averaged over the classes of wave vectors
 * whose absolute integer components are equal up to order.  The classes come
 * in order of radius; k_out[b] is the radius sqrt(i^2 + j^2 + k^2) in units of
 * the grid's wave-number step (2 pi / (n h) for n points of spacing h) and
 * s_out[b] the average.  With k_out or s_out null only *nbins is set, to the
 * number of classes; otherwise *nbins gives the capacity of both arrays and is
 * set to the number written.  Allocates device scratch; waits for the result. */
int sp_structure_factor(sp_handle* h, int inst, int field, int threshold, double* k_out,
                        double* s_out, int* nbins);

/* ---- learned jump (surrogate path) ------------------------------------------
 * No counterpart in SymPhas.  BF16 tensor-core building blocks of the
 * convolutional surrogate that jumps k steps of the finite-difference solver
 * at a time; the solver judges every jump.  All pointers are device memory,
 * activations NHWC bfloat16, work is queued on `stream` (a cudaStream_t). */
/* z / a [n][h][w][cout] = conv3x3(x [n][h][w][cin], w [cout][3][3][cin]) with
 * circular padding, + bias (fp32, or null) + res (bf16 NHWC, or null); a gets
 * gelu(z) (tanh form); either output may be null.  cin a multiple of 32, cout
 * even. */
int sp_conv3x3_fwd(const void* x, const void* w, const float* bias, const void* res, void* z,
                   void* a, int n, int h, int w_, int cin, int cout, void* stream);
/* The same convolution on the 5th-generation tensor cores (tcgen05.mma, fp32
 * accumulator in tensor memory): cin a multiple of 8, cout 32 or a multiple of
 * 64.  Its waits are bounded; a CTA that gives up sets a device flag, which
 * sp_conv_tc_status reads (after a device synchronize) and clears. */
int sp_conv3x3_fwd_tc(const void* x, const void* w, const float* bias, const void* res, void* z,
                      void* a, int n, int h, int w_, int cin, int cout, void* stream);
int sp_conv_tc_status(int* gave_up);
/* The same convolution on tcgen05 with every input pixel gathered once: the
 * input staged as a strip of circularly padded positions (one 16-byte row per
 * position and 8-channel chunk), the nine taps as start-address offsets of
 * the MMA operand, two or four 128-position accumulators per CTA in tensor
 * memory (the CTA shape is chosen per layer class; SP_STRIP_SHAPE="mt,cb,s"
 * fixes it for timing),
 * the weights re-tiled into `wt` (9 cin cout bf16 of scratch, device memory)
 * and loaded with one bulk copy per channel block.  cin a multiple of 16,
 * cout 32, 64 or a multiple of 128, w_ <= 764, bias 16-byte aligned; bounded
 * waits report through sp_conv_tc_status. */
int sp_conv3x3_fwd_strip(const void* x, const void* w, void* wt, const float* bias,
                         const void* res, void* z, void* a, int n, int h, int w_, int cin,
                         int cout, void* stream);
/* The same convolution of the nearest 2x up-sampling of x [n][h/2][w_/2][cin]
 * (h and w_ even: the output's extents), without materialising the
 * up-sampled input: the strip gather reads each position's source pixel.  No
 * counterpart in SymPhas (the jump network's decoder). */
int sp_conv3x3_fwd_strip_up2(const void* x, const void* w, void* wt, const float* bias,
                             const void* res, void* z, void* a, int n, int h, int w_, int cin,
                             int cout, void* stream);
/* dw [cout][3][3][cin] (fp32) += weight gradient of that convolution for the
 * output gradient dy [n][h][w][cout]; cin a multiple of 32, cout of 8, fewer
 * than 2^31 pixels. */
int sp_conv3x3_wgrad(const void* x, const void* dy, float* dw, int n, int h, int w_, int cin,
                     int cout, void* stream);
/* x [npix][c] (bf16) = the fp32 field psi [npix] in channel 0 and zeros in
 * the others (c a multiple of 8, x 16-byte aligned): the jump network's input
 * in one pass.  No
 * counterpart in SymPhas. */
int sp_embed_channel0_bf16(const float* psi, void* x, long long npix, int c, void* stream);
/* y [n][h/2][w_/2][c] = 2x2 average of x [n][h][w_][c] (bf16, channels last;
 * h, w_ even, c a multiple of 8, 16-byte aligned rows): the jump network's
 * pooling at inference.  No counterpart in SymPhas. */
int sp_avgpool2_bf16(const void* x, void* y, int n, int h, int w_, int c, void* stream);
/* wf [cin][3][3][cout] = w [cout][3][3][cin] rotated by 180 degrees: the input
 * gradient of the convolution is sp_conv3x3_fwd(dy, wf). */
int sp_conv3x3_flip(const void* w, void* wf, int cin, int cout, void* stream);
/* One bias-corrected Adam step (step >= 1) on n fp32 master weights w with
 * gradient g and moments m, v; writes a bf16 copy to wb when not null. */
int sp_adam_step(float* w, void* wb, const float* g, float* m, float* v, long long n, float lr,
                 float b1, float b2, float eps, int step, float weight_decay, void* stream);

/* ---- no-allocation variant of the reduction -------------------------------
 * No counterpart in SymPhas.  For callers that cannot call cudaMalloc -- an
 * application whose device memory belongs to another allocator (a framework's
 * caching pool that has reserved the GPU, a host with a fixed memory budget),
 * or a stepping loop that must not stall, as cudaMalloc and cudaFree can
 * synchronise the whole device.  Same sums as sp_reduce, but on fields the
 * caller already holds in device memory and without a handle:
 *   fields  device pointer, `batch` instances back to back, each holding the
 *           model's fields (2 for SP_MODEL_C, else 1) as compact interiors
 *           (x-fastest, periodic on every axis), dtype SP_F32 or SP_F64:
 *           batch * fields * n[0] * n[1] (* n[2]) elements, which the call
 *           cannot check;
 *   out     device pointer to 2 * batch doubles: (mass of field 0, energy)
 *           per instance; written in stream order on `stream`.  No host wait
 *           is made, so a NaN or infinite sum is written as it is (sp_reduce
 *           reports it as SP_ENONFINITE): the caller checks `out`;
 *   model, coeff, h select the free-energy density as in sp_reduce (models
 *           A, B, C, AMK, BMK; h positive and finite); energy is scaled by
 *           h^D, mass is not.
 * It calls no allocator.  Its scratch is one static device array of
 * SP_NOALLOC_MAX_INSTANCES * SP_NOALLOC_BLOCKS_PER_INSTANCE * 2 doubles
 * (128 KiB) that every GPU loading this library keeps until the process exits;
 * batch > SP_NOALLOC_MAX_INSTANCES is rejected with SP_EINVAL.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  Every call shares the
 * array: calls that overlap on the GPU (other streams, other host threads)
 * race and must be ordered by the caller. */
#define SP_NOALLOC_MAX_INSTANCES 64
#define SP_NOALLOC_BLOCKS_PER_INSTANCE 128
int sp_reduce_fields_noalloc(const void* fields, int dtype, int dim, const int n[3], int model,
                             const double coeff[8], double h, int batch, double* out,
                             void* stream);
/* Message of the last failure of sp_reduce_fields_noalloc on this thread. */
const char* sp_noalloc_error(void);

/* ---- regional systems (moving window) ---------------------------------------
 * SolverFT on SolverSystemFDwSD (sol/inc/solversystem.h:62-77): the system's
 * RegionalGrid (datatypes/inc/grid.h:2038-2158) holds only a window of the
 * domain -- select_region origin and dims in storage coordinates, each with a
 * 3-deep rim -- and reads `empty` everywhere else; the solver evaluates the
 * window's interior only, and update_regional_system
 * (sol/inc/boundarysystem.h:438-471) moves the window after the field.
 * Here the window is a handle of its own, stepped by the fused kernels: its
 * halo is the rim, holding `empty` (constant) except along an axis that the
 * window spans from origin 0, which stays periodic.  The domain itself must
 * be periodic on every side; single-field models only (SymPhas gives every
 * field of a multi-field model a window of its own).  Searches for the next
 * window run on the host over a byte mask (value >= cutoff) that a kernel
 * builds from the window, in the reference's buffer order. */
typedef struct sp_regional_params {
  double resize_delta;   /* time between window updates (params::regional_resize_time, 3.0) */
  double padding_factor; /* window / bounding box (params::regional_resize_factor, 2.0) */
  double cutoff_eps;     /* cutoff = minimum + eps (params::regional_resize_cutoff_eps, 1e-6) */
  int fixed;             /* 1: re-centre keeping the size (params::regional_resize_is_fixed);
                            0: resize to the bounding box again */
} sp_regional_params;

typedef struct sp_regional sp_regional;

/* Create a regional system over the whole domain `desc` (dim 2 or 3, batch 1,
 * periodic sides, a single-field model).  The window starts as the whole
 * domain with empty = 0 (REGIONAL_GRID_OUTER_VALUE, grid.h:2022); the first
 * update (the first step) resizes it around the values >= min + eps. */
int sp_regional_create(const sp_desc* desc, const sp_regional_params* params,
                       sp_regional** out);
/* Whole-domain interior values (x-fastest, dtype of desc) in: the window
 * takes the values at its cells. */
int sp_regional_upload(sp_regional* r, const void* host, size_t bytes);
/* Whole-domain interior values out: the window's interior, `empty` elsewhere. */
int sp_regional_download(sp_regional* r, void* host, size_t bytes);
/* `nsteps` iterations of run_model (modules-models.h:480-491): update(time)
 * -- the window check -- then equation and step, then time += dt; the steps
 * between window checks run as one sp_step of the window's handle. */
int sp_regional_step(sp_regional* r, int nsteps);
/* Move the window to origin / dims (RegionalGrid::adjust(select_region),
 * grid.h:2118-2128), dims including the rim, each at most the domain's
 * storage extent. */
int sp_regional_adjust(sp_regional* r, const int origin[3], const int dims[3]);
/* Origin and dims of the window; state = {empty, cutoff, time, next update
 * index}. */
int sp_regional_window(const sp_regional* r, int origin[3], int dims[3], double state[4]);
/* Change the time step of further sp_regional_step calls (the present
 * window's handle and every window handle made later). */
int sp_regional_set_dt(sp_regional* r, double dt);
/* Run the regional system's work on `stream` (a cudaStream_t): the present
 * window's handle and every window handle made later. */
int sp_regional_set_stream(sp_regional* r, void* stream);
/* The window's handle (null while the window has no interior): for
 * sp_kernel_info, sp_launch_count, sp_set_stream and the like. */
sp_handle* sp_regional_handle(sp_regional* r);
const char* sp_regional_error(const sp_regional* r);
void sp_regional_destroy(sp_regional* r);
/* The window search alone, on the host (no GPU needed): the window after a
 * re-centre (mode 0, grid::adjust_region) or a resize (mode 1,
 * grid::resize_adjust_region with `factor` and `rel_eps`) of the window
 * (origin, dims) of a domain with storage extents G, given the byte mask of
 * the window's buffer (dims[0]*dims[1]*dims[2] bytes, x-fastest, rim
 * included, nonzero where value >= cutoff). */
int sp_region_search(int dim, const int G[3], const int origin[3], const int dims[3],
                     const unsigned char* mask, int mode, double factor, double rel_eps,
                     int new_origin[3], int new_dims[3]);

const char* sp_last_error(const sp_handle* h);
/* Message of the last failure of sp_create (no handle exists then). */
const char* sp_create_error(void);
void sp_destroy(sp_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* SYMPHAS_B200_H */
