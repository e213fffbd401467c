/* simson_b200: B200-native time step of Simson's bla (temporal channel).
 *
 * C ABI of the drop-in for the two plane loops of the reference driver:
 *   bla/bla.f:2251-2290  do ybp: call nonlinbl(...)   -> sgpu_nonlin
 *   bla/bla.f:2433-2476  do zbp: call linearbl(...)   -> sgpu_linear
 * plus the startup partial right-hand side bla/bla.f:1562 (prhs) -> sgpu_prhs.
 *
 * Calling convention: plain C, every entry returns 0 on success or a negative
 * SGPU_E* code (the Fortran shim maps non-zero to stopnow(code)).  Arrays use
 * the reference's main-storage layout ur(memnx,memny,memnz,slot), 0-based
 * index x + memnx*(y + memny*(z + memnz*slot)), split real/imaginary double
 * arrays exactly as bla keeps them (bla/bla.f:67, bla/par.f:111-120).  Slots:
 * 0-2 u,v,w and 3-4 omega_x,omega_z (Fourier x/z, physical y), 5-6 the partial
 * right-hand sides p_v, p_omega_y (Chebyshev y).
 *
 * Ownership: the device owns the state between upload and download; one
 * context per process, not re-entrant, called from one host thread.
 */
#ifndef SIMSON_B200_H
#define SIMSON_B200_H

#include <stddef.h> /* size_t */

#ifdef __cplusplus
extern "C" {
#endif

#define SGPU_OK 0
#define SGPU_E_PARAM (-1)      /* invalid parameters (grid, nst, dt, ...) */
#define SGPU_E_CUDA (-2)       /* CUDA runtime error (allocation, launch)  */
#define SGPU_E_STATE (-3)      /* call out of order (no state uploaded)    */
#define SGPU_E_CFL (-4)        /* CFL*dt > 10: the reference stops (wcflbl.f:93) */
#define SGPU_E_NAN (-5)        /* non-finite value detected in the state   */
#define SGPU_E_TIMEOUT (-6)    /* a bounded device wait ran out (a lost completion) */

#define SGPU_FP64 0            /* every transform and solve in FP64 */
#define SGPU_MIXED 1           /* FP32 x/z FFTs, products, Chebyshev transforms and u,v,w,omega
                                  storage; FP64 tau solves, mean flow, p_v/p_omega and prhs */

typedef struct sgpu_ctx sgpu_ctx;

/* The subset of par.f and bla.i that the channel step reads. */
typedef struct sgpu_params {
  int nx, ny, nz;   /* par.f nx, ny, nz (nfxd = nfzd = 1, nfyd = 0) */
  double re;        /* bla.i re (centreline Reynolds number) */
  double xl, zl;    /* box length in x and z */
  double dt;        /* time step (bla.i dt > 0; a variable step: sgpu_set_dt) */
  int nst;          /* RK stages: 3 or 4 (bla.i nst; bla/rkcoeff.f) */
  int cflux;        /* 1: constant mass flux (bla.i cflux); 0: fixed px */
  double mflux;     /* target flux under cflux (bla.f:1629 sets 4/3) */
  double px;        /* pressure gradient; first guess under cflux (-2/re) */
  double rot;       /* bla.i rot */
  int icfl;         /* CFL every icfl substeps (bla.i icfl, rounded as rparambl.f:1862) */
  int precision;    /* SGPU_FP64 or SGPU_MIXED */
  int device;       /* CUDA device ordinal */
} sgpu_params;

/* bla/bla.f:709-1082 subset: allocate the resident state and tables.
 * Replaces the preprbl/rkcoeff set-up for the device path. */
int sgpu_init(const sgpu_params* prm, sgpu_ctx** ctx);
int sgpu_finalize(sgpu_ctx* ctx);

/* Host <-> device state in the reference layout (bla/par.f:111-120).
 * nslots = number of leading slots transferred (3: velocities only). */
int sgpu_upload_state(sgpu_ctx* ctx, const double* ur, const double* ui, int nslots);
int sgpu_download_state(sgpu_ctx* ctx, double* ur, double* ui, int nslots);
/* Mean-flow partial right-hand side puw(ny,2) (linearbl.f argument puw). */
int sgpu_upload_puw(sgpu_ctx* ctx, const double* puw);
int sgpu_download_puw(sgpu_ctx* ctx, double* puw);

/* bla/prhs.f, called at bla/bla.f:1562: from u,v,w (slots 0-2) build
 * omega_x, omega_z, p_v, p_omega and puw for the first stage; also resets the
 * RK bookkeeping to the first substep (bla/bla.f:1464-1478, 1622-1662). */
int sgpu_prhs(sgpu_ctx* ctx);

/* One RK substep, split like the reference driver:
 * sgpu_nonlin replaces the nonlinbl plane loop (bla/bla.f:2251-2290,
 * bla/nonlinbl.f:9-32) including boxcfl (CFL partial maxima);
 * sgpu_linear replaces the RK-weight update (bla/bla.f:2384-2397) and the
 * linearbl plane loop (bla/bla.f:2433-2476, bla/linearbl.f:9-27), including
 * the constant-flux px correction, and advances it/t (bla/bla.f:2598-2607). */
int sgpu_nonlin(sgpu_ctx* ctx);
int sgpu_linear(sgpu_ctx* ctx);
/* nsub consecutive substeps (nonlin + linear), enqueued without host syncs
 * (nst substeps per full step). */
int sgpu_step_rk(sgpu_ctx* ctx, int nsub);

/* Variable time step (bla.i dt <= 0; the reference's vart).  sgpu_cfl_rate
 * gives the CFL number per unit time step of the current state, as
 * bla/getdt.f forms it (pi times the maximum over the planes of
 * |u|/dx + |v|/dy + |w|/dz, bla/boxcfl.f, plus 2 |rot|; the first step's dt
 * is cflmax over it); it synchronises and leaves the state unchanged.
 * sgpu_set_dt sets the time step of the next full step (the reference's dtnp1,
 * bla/bla.f:2358-2372): called before a step's last substep, it enters that
 * substep's weights of the next stage (:2389-2397) and becomes the step's
 * successor's dt (:2610); called before sgpu_prhs, it is the first step's
 * dt.  Without it the step stays sgpu_params.dt.  Not on a shard. */
int sgpu_cfl_rate(sgpu_ctx* ctx, double* rate);
int sgpu_set_dt(sgpu_ctx* ctx, double dt);

/* Scalars, in this order: px, mflux, t, cfl (CFL*dt of the last evaluated
 * substep, wcflbl.f), an, bn, anp1, bnp1, cnp1, it, tc, dt.  Synchronises.
 * Returns SGPU_E_CFL when CFL*dt > 10 (the reference's stop, wcflbl.f:93)
 * and SGPU_E_NAN when px or the mass flux is not finite (a non-finite value
 * anywhere in u, v, w reaches them within one substep), SGPU_E_TIMEOUT when a
 * bounded wait of a tensor-core kernel ran out since the last call (see
 * sgpu_set_wait_limit); the driver calls it after each step it checks, as
 * the reference checks every icfl substeps. */
int sgpu_get_scalars(sgpu_ctx* ctx, double* out, int n);

/* Large-eddy model, the reference's sgs.i (bla/rparamles.f:31-60):
 *   iles        0 none, 1 ADM-RT (approximate deconvolution, relaxation term),
 *               2 eddy viscosity (Smagorinsky; dynamic when cs = 0),
 *               3 HPF eddy viscosity (Smagorinsky on the high-pass filtered field)
 *   cutoff_inv  1 / cut-off wavenumber fraction of the primary filter (1.5)
 *   iord        order N of the deconvolution, 0..5 (5)
 *   chi         relaxation coefficient (0.2)
 *   ihighorder  0 two-dimensional, 1 iterative, 2 tensorial filtering (2)
 *   cs          Smagorinsky constant; 0 = dynamic procedure (0)
 *   ineg        dynamic coefficient: 0 no clipping, 1 C >= 0, 2 nu_t + nu >= 0 (1) */
typedef struct {
  int iles;
  double cutoff_inv;
  int iord;
  double chi;
  int ihighorder;
  double cs;
  int ineg;
} sgpu_les_params;

/* Enables the LES model (rparamles + bla/bla.f:1489-1518).  Call after
 * sgpu_init and before sgpu_prhs.
 * iles = 1: builds the filters of bla/init_filter.f; sgpu_prhs filters the
 *   start-up velocities (bla/prhs.f:95-193), step 2 adds -chi gu
 *   (bla/nonlinbl.f:920-965), step 3 refilters (bla/linearbl.f:1871-1960).
 * iles = 2: every substep starts with the SGS stress of bla/les.f and its
 *   divergence (bla/sgs_stress.f, the loops of bla/bla.f:1945-2020); step 2
 *   adds -sigma (bla/nonlinbl.f:1011-1048).  Needs nx, nz divisible by 4.
 * iles = 3: the high-pass filter of iles = 1 applied to u, v, w, omega_x,
 *   omega_z after prhs and every step 3 (bla/prhs.f, bla/linearbl.f:
 *   1871-2060), and every substep the eddy-viscosity stress of iles = 2
 *   formed with the strain of the filtered field (bla/les.f:404-450,
 *   883-966): cs > 0 fixed (ineg = 1), or cs = 0 the dynamic HPF
 *   procedure (bla/les.f:968-1383): a secondary filter with the x/z transfer
 *   functions over a quarter of the wavenumbers (bla/bla.f:1520-1545) on the
 *   same five fields, L_ij from the resolved velocity, M_ij from the strain
 *   of the primary filtered field and the test-filtered strain of the
 *   secondary one, the coefficient as for iles = 2 (ineg 0, 1, 2). */
int sgpu_set_les(sgpu_ctx* ctx, const sgpu_les_params* p);

/* gur, gui(memnx, memny, memnz, 1..3): the filtered velocities (iles = 1, and
 * iles = 3 after sgpu_prhs or a step 3) or the SGS force sigma (iles = 2, 3
 * after a step 2). */
int sgpu_download_les(sgpu_ctx* ctx, double* gr, double* gi);

/* taur, taui(memnx, memny, memnz, 1..6) (iles = 2): the SGS stress of the
 * last substep, components 11 12 13 22 23 33 (bla/les.f:1620-1640). */
int sgpu_download_sgs_stress(sgpu_ctx* ctx, double* tr, double* ti);

/* Learned SGS model (no counterpart in the reference): an MLP from the
 * resolved velocity gradient and the wall distance to the SGS stress,
 *   x_(3i+j) = s_in du_i/dx_j,  x_9 = s_y (1 - |y|)
 *   tau = s_out (W3 tanh(W2 tanh(W1 x + b1) + b2) + b3)
 * (w1 [64][10], w2 [64][64], w3 [6][64] row-major, biases b1[64], b2[64],
 * b3[6]; tau components 11 12 13 22 23 33).  Weights and activations are
 * used in BF16 with FP32 accumulation.  The stress takes the place of the
 * eddy-viscosity stress (bla/les.f:1620-1640): its divergence is formed as
 * bla/sgs_stress.f does and subtracted from H in step 2. */
typedef struct {
  const float *w1, *b1, *w2, *b2, *w3, *b3;
  float s_in, s_y, s_out;
} sgpu_sgs_mlp;

/* Enables the learned model for the following substeps (replaces any LES
 * model set with sgpu_set_les).  Needs nx, nz divisible by 4. */
int sgpu_set_sgs_mlp(sgpu_ctx* ctx, const sgpu_sgs_mlp* p);

/* Per-plane fallback of the learned model to the eddy-viscosity model (no
 * counterpart in the reference; the plain model is bla/les.f's, dynamic when
 * cs = 0, clipping ineg as in sgpu_les_params).  enable = 1: every substep,
 * after the network's stress, each xz-plane y sums P = tau_ij S_ij and |P|
 * over its points (tau the network's stress, S_ij the resolved strain rate;
 * P > 0 is backscatter, energy from the subgrid to the resolved scales) and
 * takes the eddy-viscosity stress instead when sum P > bound * sum |P|
 * (bound 1: never; bound below -1: always; 0: on net backscatter).  The
 * eddy-viscosity model runs on the switched planes only.  enable = 0: off.
 * Call after sgpu_set_sgs_mlp. */
int sgpu_set_sgs_fallback(sgpu_ctx* ctx, int enable, double bound, double cs, int ineg);

/* The plane switches of the last substep: planes[ny] (1 = eddy-viscosity
 * stress), and, if sums is not NULL, sums[2*ny] = (sum P, sum |P|) per plane.
 * Synchronises the library's stream.  SGPU_E_STATE before the fallback was
 * enabled once. */
int sgpu_sgs_fallback_planes(sgpu_ctx* ctx, int* planes, double* sums);

/* Training of the learned SGS model (no counterpart in the reference):
 * iters full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8, learning
 * rate lr; *adam_step counts the steps taken, for the bias corrections) on
 * the mean squared error sum (y - t)^2 / (6 n) of the network of
 * sgpu_sgs_mlp without its scales, y = W3 tanh(W2 tanh(W1 x + b1) + b2) + b3,
 * over n samples x[n][10], t[n][6] (host arrays, e.g. the features and
 * targets of sgpu_box_filter_sample, scaled as they will be at inference).
 * params: the 5254 FP32 weights packed W1 [64][10], b1 [64], W2 [64][64],
 * b2 [64], W3 [6][64], b3 [6]; adam_m, adam_v the same size; all three are
 * updated.  On return *loss (if not NULL) holds the loss and grad (if not
 * NULL, 5254 values) the gradient at the final weights (iters = 0: at the
 * given ones).  FP32 arithmetic; allocates its device buffers for the call.
 * Synchronises the library's stream. */
int sgpu_sgs_mlp_train(sgpu_ctx* ctx, float* params, float* adam_m, float* adam_v, int* adam_step,
                       const float* x, const float* t, long long n, int iters, float lr, float* loss,
                       float* grad);

/* The MLP alone on n feature rows: x[n][10] -> y[n][6] (host arrays), the
 * same tensor-core kernel the step runs.  Loads p's weights. */
int sgpu_sgs_mlp_eval(sgpu_ctx* ctx, const sgpu_sgs_mlp* p, const float* x, float* y, long long n);

/* Statistics of the current state, as bla/boxamp.f and bla/wampbl.f:124-278
 * compute them at the start of a full step when iamp > 0: amp[20*ny] in the
 * layout of amp(nyp,20) (plane averages of squared velocity and vorticity
 * fluctuations, <|omega_y|^2/k^2>, Reynolds stresses, mean U, W, Omega_x,
 * Omega_z per y; column 13 unused), and, if row is not NULL, the 19 values of
 * one amp.stat line (bla/wampbl.f:276-278): t, u/v/w rms, omega_x/y/z rms,
 * <|omega_y|^2/k^2>, <u'v'>, e0, h+ (Re_tau), px, Re_bulk, wall shears tau1
 * (y=+1) and tau2 (y=-1), 99 %, displacement and momentum thickness, W bulk.
 * Synchronises the library's stream. */
int sgpu_amplitudes(sgpu_ctx* ctx, double* amp, double* row);

/* xy statistics (bla/boxxys.f, taken by bla/bla.f:2069-2107 at the start of a
 * step when mod(it-1-nst, ixys) = 0 and t >= txys; the caller decides when):
 * one sample of the current state with weight dtn is added to the running
 * sums xys and sumw (sumw += dtn), on the library's stream.  Entries computed
 * (1-based, the reference's numbering): 1-15 means and second moments of
 * u_i, omega_i and uv, uw, vw; 25-30 the dissipation tensor du_i/dx_k
 * du_j/dx_k; 43-44 running min / max over z of u - <u>_z; 45-51 S_ij S_ij
 * and S_ij; 63-72 third moments; 75-77 u_i^4.  When sgpu_pressure has
 * been called on the current state (the reference needs the pressure of the
 * sampled state, bla/bla.f:1833-1840), also the pressure entries 31-42,
 * 73-74, 78-79; any step or upload makes that pressure stale.  LES and MHD
 * entries stay zero.  nx <= 512.  Not on a shard. */
int sgpu_xys_sample(sgpu_ctx* ctx, double dtn);

/* The running sums: xys[96*ny*nx] in the layout of the reference's
 * xys(nx, ny, 96) (x fastest), *sumw the accumulated weight (either may be
 * read before any sample: zeros).  Synchronises the library's stream. */
int sgpu_xys_get(sgpu_ctx* ctx, double* xys, double* sumw);

/* Zero the running sums (a new averaging period, bla/bla.f:1573). */
int sgpu_xys_reset(sgpu_ctx* ctx);

/* Pressure of the current state, as bla/bla.f:2486-2527 computes it after a
 * step whose field is saved (bla/nonlinp.f, bla/linearp.f: the Poisson
 * equation with the Neumann conditions of the wall-normal momentum equation,
 * the mean mode by integration of H2): p in the layout of one slot of ur, ui
 * (Fourier x/z, physical y; the kz = -nz/2 plane is zero).  The state is not
 * changed.  FP64 arithmetic; under SGPU_MIXED from the FP32 state.
 * Synchronises the library's stream.  Not on a shard. */
int sgpu_pressure(sgpu_ctx* ctx, double* pr, double* pi);

/* Training sample for the learned SGS stress (sgpu_set_sgs_mlp) from the
 * resolved state.  No reference counterpart (the reference's dynamic model
 * forms the analogous filtered products internally with a spectral cut-off,
 * bla/les.f:709-881): here a top-hat box filter over cells of f x f points of
 * the nx x nz grid (f divides nx and nz; y unfiltered).  Per point of the coarse grid
 * (ny x nz/f x nx/f, x fastest): features[10] = the nine filtered velocity
 * gradients du_i/dx_j (i-major) and the wall distance 1 - |y|, targets[6] =
 * tau_ij = <u_i u_j> - <u_i><u_j> (11 12 13 22 23 33), float.  Synchronises
 * the library's stream.  Not on a shard. */
int sgpu_box_filter_sample(sgpu_ctx* ctx, int factor, float* features, float* targets);

/* The driver keeps the state: advance it by nsteps RK3 steps, each step
 * uploading all 7 slots from ur, ui (reference layout, as sgpu_upload_state;
 * pinned host memory for full speed) and downloading the result into them
 * (as sgpu_download_state), so the host arrays are current after every step.
 * The copies of consecutive steps are pipelined: each slot moves in eight
 * pieces, and a piece of step n+1's upload waits only for the same piece of
 * step n to be back on the host, overlapping the rest of the download (PCIe
 * is full duplex).  Without LES, the first substep's nonlinear step starts
 * once slots 0-4 are on the device, while p_v and p_omega still upload.
 * Returns after the last download.  Not on a shard. */
int sgpu_offload_steps(sgpu_ctx* ctx, double* ur, double* ui, int nsteps);

/* Multi-GPU runs (one context per GPU, the reference's MPI decomposition of
 * bla/par.f:102 and bla/getpxz.f / putpxz.f mapped to whole-state contexts):
 * restrict this context to a shard -- step 2 (sgpu_nonlin) on the xz-planes
 * ylo <= y < yhi, step 3 (sgpu_linear) on the kz planes zlo <= iz < zhi (iz
 * the stored kz index, kx all).  (0, ny, 0, nz) is the whole domain.  Before
 * step 2 each shard needs slots 0-4 of its planes from every shard's kz
 * planes, after it each shard needs slots 0-2 (H) of its kz planes from every
 * shard's planes; the host moves these blocks (sgpu_copy_block plus its
 * transport, e.g. an NCCL all-to-all).  sgpu_prhs still works on the whole
 * uploaded state; LES and sgpu_amplitudes need the whole domain
 * (SGPU_E_PARAM / SGPU_E_STATE on a shard), and so does sgpu_step_rk (the
 * exchanges sit between its two steps).  Replaces the plane transposes of
 * bla/getpxz.f:127-149 and bla/putpxz.f:69-93. */
int sgpu_set_shard(sgpu_ctx* ctx, int ylo, int yhi, int zlo, int zhi);

/* Copy state slots slot0 .. slot0+nslots-1 of the planes ylo..yhi-1 and kz
 * planes zlo..zhi-1 between the state and the device buffer buf (to_state =
 * 0: state -> buf, 1: buf -> state), packed as [slot][y][kz][kx] in the
 * state's storage (complex FP32 for slots 0-4 under SGPU_MIXED, complex FP64
 * otherwise); *bytes receives the block size (buf == NULL only reports it).
 * Synchronises. */
int sgpu_copy_block(sgpu_ctx* ctx, int slot0, int nslots, int ylo, int yhi, int zlo, int zhi, void* buf,
                    int to_state, size_t* bytes);
/* OR'ed into sgpu_copy_block's to_state: only enqueue the copy on the
 * library's stream (sgpu_stream), without synchronising; the transport of the
 * blocks (e.g. NCCL) is then ordered on the same stream. */
#define SGPU_BLOCK_NOSYNC 2

/* The library's CUDA stream (a cudaStream_t), for work that a host orders
 * with the step's kernels. */
int sgpu_stream(sgpu_ctx* ctx, void** stream);

/* Sharded runs: the CFL number needs the maximum over all shards, as the
 * reference all-reduces it over its MPI ranks (bla/wcflbl.f:82-85) before its
 * stop test (:93).  On a shard, sgpu_nonlin and sgpu_get_scalars leave that
 * test to the host: sgpu_cfl_partial gives this shard's partial maximum
 * max(|u|/dx + |v|/dy + |w|/dz) of the last substep that evaluated it and
 * *pending = 1 if it has not been reduced yet (then it synchronises; with
 * *pending = 0 it returns 0 at once);
 * sgpu_cfl_set_global takes the maximum over the shards, forms CFL*dt
 * (bla/wcflbl.f:87) and returns SGPU_E_CFL (above 10) or SGPU_E_NAN. */
int sgpu_cfl_partial(sgpu_ctx* ctx, double* cflp, int* pending);
int sgpu_cfl_set_global(sgpu_ctx* ctx, double cflp);

/* Step 3's pencil kernel: warp = 1 solves each (kx, kz) pencil with one warp
 * (every column of the pencil in registers across the warp: the tau solves
 * by the partition method with a parallel cyclic reduction over the lanes,
 * the Chebyshev derivatives as warp scans), warp = 0 with one thread per
 * pencil sweeping its columns through memory in the reference's elimination
 * order (bla/trid.f:120-200), warp = 2 chooses: the warp kernel up to 8192
 * pencils (nz nx/2; grids such as the LES grid 64x97x64, where one thread
 * per pencil leaves the GPU idle), the thread kernel above (the default,
 * also set at sgpu_init; SIMSON_PENCIL_WARP=0/1 in the environment forces
 * one for new contexts).  Both solve the same tau systems, to round-off.
 * SGPU_E_PARAM for warp = 1 when ny > 256. */
int sgpu_set_pencil_kernel(sgpu_ctx* ctx, int warp);

/* Failure detection of the tensor-core kernels (the mixed path's Chebyshev
 * transforms and the learned SGS model): every wait of theirs on an mbarrier
 * is bounded.  limit: iterations of each wait in their main loops (0: the
 * default, 2^20); a wait that runs out makes the kernel let its own copies
 * and MMAs in flight finish (with the default limit), free its tensor memory
 * and return, and the next sgpu_get_scalars (or sgpu_sgs_mlp_eval) returns
 * SGPU_E_TIMEOUT once; the state of that substep is not valid (upload it
 * again).  test_timeout = 1 makes the first wait of every such launch wait on
 * a barrier that nothing completes, so that the timeout path can be tested
 * without a fault; 0 turns that off.  The reference has no counterpart (its
 * stopnow codes, bla/stopnow.f, stop the run). */
int sgpu_set_wait_limit(sgpu_ctx* ctx, int limit, int test_timeout);

/* Stream-ordered timing on the library's stream: record event slot (0..15),
 * elapsed milliseconds between two recorded slots (synchronises on b). */
int sgpu_event_record(sgpu_ctx* ctx, int slot);
int sgpu_event_elapsed(sgpu_ctx* ctx, int a, int b, float* ms);
int sgpu_sync(sgpu_ctx* ctx);

/* No counterpart in the reference.  The nonlinear step of sgpu_nonlin for
 * callers that cannot let the library allocate device memory: hosts that own
 * every device buffer themselves (a Fortran/OpenACC code with its own memory
 * pool, or one that has already reserved the GPU's memory for its fields).
 * fields_in: device array of u, v, w, omega_x, omega_z, each ny x nz x nx/2
 * complex doubles (kx fastest, the library's device layout); h_out: device
 * array of H1, H2, H3 in the same layout; cflp_max (host, may be NULL): the
 * CFL partial maximum max|u|/dx+|v|/dy+|w|/dz of bla/boxcfl.f; stream: a
 * cudaStream_t or NULL.  prm->precision must be SGPU_FP64 (the arrays are
 * complex doubles); no LES term is added.  Allocates nothing: the step's
 * intermediates sit in one static device array of 64 MiB that every GPU
 * loading the library holds until exit; grids needing more
 * (9*ny*(3nz/2)*(nx/2)*16 bytes) are rejected with SGPU_E_PARAM.  Every call
 * shares that array, so calls that overlap on the GPU race.  Every call looks
 * up the array's device address with the caller's device current (the first
 * lookup on a device may load the library's device code: make the first call
 * on a device before any stream capture), copies its small tables from host
 * memory into the array, and, when cflp_max is given, waits for the stream to
 * read the CFL maximum back. */
int sgpu_nonlin_noalloc(const sgpu_params* prm, const void* fields_in, void* h_out, double* cflp_max,
                        void* stream);

/* Spatial simulation (bla.i spat = .true.) in the channel (ibc = 0; the
 * spatially developing Poiseuille and Couette flows, fltype 4 and 5): the
 * fringe forcing of bla/fring.f (no wave, streak or Orr-Sommerfeld forcing),
 * H -= lambda(x) (u - U_b(x, y)) on the three components in physical space
 * after the products of step 2 (bla/nonlinbl.f:681-691), and the same on the
 * products of sgpu_pressure (bla/fringp.f).  The host computes the base flow
 * (bla/bflow.f) and the pressure gradient (bla/bla.f:1655-1661: px = 0 and no
 * constant flux outside the temporal channel). */
typedef struct {
  double fstart, fend; /* bla.i fstart, fend: the fringe's start and end in x */
  double frise, ffall; /* bla.i frise, ffall: its rise and fall distances */
  double fmax;         /* bla.i fmax: its strength (0: no fringe) */
  double xsc;          /* x of the frame (bla/bla.f:1819 xs - cnp1 u0low; 0 without Galilean shift) */
} sgpu_fringe;

/* lambda at the nxp physical x points (x point 2k-2 and 2k-1 are the
 * reference's fring1(k), fring2(k)), as bla/ffun.f:58-83 computes it with the
 * smooth step of bla/step.f; zero outside the fringe.  Host only (no context,
 * no GPU).  SGPU_E_PARAM when the fringe leaves the box. */
int sgpu_fringe_function(const sgpu_fringe* f, int nxp, double xl, double* lambda);

/* Fringe forcing from now on (f == NULL or fmax == 0: off), towards the base
 * flow of sgpu_set_base_flow (zero until set).  Replaces bla/bla.f:2166-2175
 * (ffun) and the fring call of bla/nonlinbl.f:681-691. */
int sgpu_set_fringe(sgpu_ctx* ctx, const sgpu_fringe* f);

/* The base flow bu1, bu2(nxp/2+1, nyp, 3) of bla/bflow.f (u, v, w in
 * physical space at the even and odd x points, the reference's x pairs; the
 * last x row is not read).  bu1 = bu2 = NULL: zero. */
int sgpu_set_base_flow(sgpu_ctx* ctx, const double* bu1, const double* bu2);

/* Per-kernel timing for profiling runs: enable, run substeps, read the
 * milliseconds and launch counts per kernel id (0 zinv, 1 xpass, 2 zfwd,
 * 3 Chebyshev forward, 4 pencil solve, 5 mean flow, 6 Chebyshev inverse,
 * 7 other).  Adds an event record per launch; not for timed runs. */
int sgpu_profile(sgpu_ctx* ctx, int enable);
int sgpu_profile_read(sgpu_ctx* ctx, double* ms, int* count, int n);

/* Page-locked host buffers for the host<->device state copies (cudaHostAlloc):
 * a Fortran host can keep ur/ui in them to get full-bandwidth transfers. */
int sgpu_host_alloc(unsigned long long bytes, void** ptr);
int sgpu_host_free(void* ptr);

/* Device kernels launched by this context so far (launch accounting). */
long long sgpu_launch_count(sgpu_ctx* ctx);
const char* sgpu_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif
