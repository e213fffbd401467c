/* Harness around the translated reference (oracle/_ref/<grid>/ref_gen.c).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, bench.py's CPU-baseline arm and
 * __graft_entry__.smoke() as the checker, never by the product.
 *
 * It plays the part of the reference driver bla/bla.f for the temporal channel
 * (fltype=1, nst=3 RK3/CN, fixed dt, ibc=0, tau method, constant mass flux,
 * no LES, no scalar, nproc=1): it sets the bla.i-level scalars that the
 * channel case uses, then runs the translated statement ranges of bla.f in the
 * order the reference time loop does (bla/bla.f:1790-2610).  The translated
 * ranges are the reference's own statements; only the glue (parameter values,
 * slot copies, the full-step time update bla/bla.f:2600-2607) is written here.
 */
#include "ref_gen.c"

#include <string.h>

void f77_stop(int code) {
  fprintf(stderr, "oracle: reference STOP %d\n", code);
  abort();
}

void f_stopnow(int *code) {
  fprintf(stderr, "oracle: reference stopnow(%d)\n", *code);
  abort();
}

static int sref_threads = 1;

/* dims[0..11] = nx ny nz nxp nyp nzp memnx memny memnz memnxyz nthread nby */
void sref_dims(int *dims) {
  dims[0] = v_nx; dims[1] = v_ny; dims[2] = v_nz;
  dims[3] = v_nxp; dims[4] = v_nyp; dims[5] = v_nzp;
  dims[6] = v_memnx; dims[7] = v_memny; dims[8] = v_memnz; dims[9] = v_memnxyz;
  dims[10] = v_nthread; dims[11] = v_nby;
}

/* Sets up the channel case; mirrors what rparambl/bla.f would leave in place
 * for a bla.i with: fltype=1, nst=3, fixed dt, ibc=0, cim=.false., cflux,
 * icfl=nst, iamp=iext=ixys=0 (disabled), iles=0, rot=0. */
int sref_setup(double re, double xl, double zl, double dt, int cflux, int icfl, int nthreads) {
  static int allocated = 0;
  if (allocated) f77_main_free();
  f77_main_alloc();
  allocated = 1;
  sref_threads = nthreads < 1 ? 1 : (nthreads > v_nthread ? v_nthread : nthreads);
#ifdef _OPENMP
  omp_set_num_threads(sref_threads);
#endif
  v_re = re; v_xl = xl; v_zl = zl;
  v_dtn = dt; v_dtmax = 1.0e30; v_vart = 0;
  v_nst = 3; v_fltype = 1; v_pert = 0; v_lin = 0; v_spat = 0;
  v_cflux = cflux ? 1 : 0;
  v_ibc = 0; v_cim = 0; v_icorr = 0;
  v_icfl = icfl; v_iamp = -1000000; v_iext = -1000000; v_ixys = -1000000;
  v_iles = 0; v_isfd = 0; v_imhd = 0; v_wbci = 0; v_loctyp = 0; v_tripf = 0;
  v_osmod = 0; v_streak = 0; v_bf3 = 0; v_do_press_nl = 0; v_do_press = 0;
  v_rot = 0.0; v_dstar = 1.0; v_my_node = 0;
  v_u0low = 0.0; v_u0upp = 0.0; v_w0low = 0.0; v_w0upp = 0.0; v_du0upp = 0.0;
  v_vsuc = 0.0; v_x0 = 0.0; v_cdev = 0.0; v_xs = 0.0; v_zs = 0.0; v_t = 0.0;
  bla_rkcoeff();
  bla_preprbl();
  bla_firststep();
  return 0;
}

/* As sref_setup for a bla.i with nst = 3 or 4 stages and, when dt <= 0, the
 * variable time step: what rparambl.f:1995-2017 leaves (vart = dt <= 0, dtmax
 * = -dt for dt < 0, cflmax = cflmaxin sqrt(3) or sqrt(8)), the save time and
 * tmax that bound the step (bla.f:2356-2380; here one far save time).  With
 * vart the first step's dt comes from getdt when sref_start runs. */
static int sref_defer_first = 0;
int sref_setup_rk(double re, double xl, double zl, double dt, int cflux, int icfl, int nthreads, int nst,
                  double cflmaxin, double tmax) {
  sref_setup(re, xl, zl, dt > 0 ? dt : 1.0, cflux, icfl, nthreads);
  v_nst = nst;
  v_vart = dt <= 0.0;
  v_dtmax = dt < 0.0 ? -dt : 1.0e30;
  v_cflmax = cflmaxin * sqrt(nst == 3 ? 3.0 : 8.0);
  v_tmax = tmax;
  v_isave = 1;
  v_tsave[0] = 1.0e30;
  v_dtn = dt > 0 ? dt : 0.0;
  bla_rkcoeff();
  sref_defer_first = v_vart;
  if (!v_vart) bla_firststep();
  return 0;
}

static long slot_size(void) { return (long)v_memnx * v_memny * v_memnz; }

void sref_set_slot(int slot, const double *re_part, const double *im_part) {
  long n = slot_size();
  memcpy(v_ur + (long)(slot - 1) * n, re_part, n * sizeof(double));
  memcpy(v_ui + (long)(slot - 1) * n, im_part, n * sizeof(double));
}

void sref_get_slot(int slot, double *re_part, double *im_part) {
  long n = slot_size();
  memcpy(re_part, v_ur + (long)(slot - 1) * n, n * sizeof(double));
  memcpy(im_part, v_ui + (long)(slot - 1) * n, n * sizeof(double));
}

/* Startup: partial right-hand side from the velocities (bla/bla.f:1562) and
 * the channel pressure-gradient / mass-flux initialisation (:1622-1662). */
void sref_start(void) {
#ifdef _OPENMP
  omp_set_num_threads(sref_threads);
#endif
  if (sref_defer_first) {
    bla_getdt();
    bla_firststep();
    sref_defer_first = 0;
  }
  bla_prhs();
  bla_pxinit();
  v_it = 1;
}

/* Spatial simulation in the channel (bla.i spat = .true., ibc = 0) with the
 * flow type of the initial field (4 Poiseuille, 5 Couette): the fringe
 * parameters of bla.i (rparambl.f leaves them as given; no wave, streak or
 * OS forcing, rbfl = .false.), then the base-flow block of bla/bla.f:1338-1374
 * (bflow, the boundary values for ibc = 0).  The pressure gradient follows
 * from bla_pxinit in sref_start (px = 0, no constant flux for fltype != 1);
 * each substep computes the fringe function (bla/bla.f:2166-2175) before
 * step 2.  Call after sref_setup / sref_setup_rk, before sref_start. */
void sref_set_spatial(int fltype, double fstart, double fend, double frise, double ffall, double fmax) {
  v_spat = 1; v_fltype = fltype; v_rbfl = 0; v_tabfre = 0; v_pert = 0; v_bf3 = 0;
  v_fstart = fstart; v_fend = fend; v_frise = frise; v_ffall = ffall; v_fmax = fmax;
  v_ampob = 0.0; v_amp2d = 0.0; v_osmod = 0; v_streak = 0; v_waves = 0;
  v_bstart = 0.0; v_blength = 0.0;
  bla_bflow();
}

/* The fringe function fring1, fring2 (nxp/2 each) at the current substep's
 * frame (bla/ffun.f), and the base flow bu1, bu2 (nxp/2+1, nyp, 3). */
void sref_get_fringe(double *f1, double *f2) {
  bla_boxshift();
  bla_ffun();
  memcpy(f1, v_fring1, (size_t)(v_nxp / 2) * sizeof(double));
  memcpy(f2, v_fring2, (size_t)(v_nxp / 2) * sizeof(double));
}
void sref_get_base(double *b1, double *b2) {
  const size_t n = (size_t)(v_nxp / 2 + 1) * v_nyp * 3;
  memcpy(b1, v_bu1, n * sizeof(double));
  memcpy(b2, v_bu2, n * sizeof(double));
}

/* One RK substep: step 2 (nonlinbl over xz-planes), CFL, RK weights, step 3
 * (linearbl over xy-planes), iteration counter and full-step time update. */
void sref_substep(void) {
#ifdef _OPENMP
  omp_set_num_threads(sref_threads);
#endif
  bla_substep_time();
  bla_boxshift();
  if (v_spat) bla_ffun();
  bla_les();
  bla_nonlin();
  bla_cfl();
  bla_vart();
  bla_rkweights();
  bla_linear();
  bla_itinc();
  if ((v_it - 1) % v_nst == 0) {
    v_t = v_t + v_dtn;
    if (v_vart) v_dtn = v_dtnp1; /* bla/bla.f:2610 */
  }
}

/* Only step 2 or only step 3 (for per-kernel parity tests). */
void sref_nonlin_only(void) {
  bla_substep_time();
  bla_boxshift();
  if (v_spat) bla_ffun();
  bla_les();
  bla_nonlin();
}
void sref_linear_only(void) {
  bla_cfl();
  bla_vart();
  bla_rkweights();
  bla_linear();
  bla_itinc();
  if ((v_it - 1) % v_nst == 0) {
    v_t = v_t + v_dtn;
    if (v_vart) v_dtn = v_dtnp1;
  }
}

/* scalars: 0 px, 1 mflux, 2 t, 3 cfl, 4 an, 5 bn, 6 anp1, 7 bnp1, 8 cnp1, 9 it, 10 tc, 11 dtn */
void sref_scalars(double *s) {
  s[0] = v_px; s[1] = v_mflux; s[2] = v_t; s[3] = v_cfl;
  s[4] = v_an; s[5] = v_bn; s[6] = v_anp1; s[7] = v_bnp1; s[8] = v_cnp1;
  s[9] = v_it; s[10] = v_tc; s[11] = v_dtn;
}

/* partial RHS of the mean flow, puw(ny, 2) */
void sref_get_puw(double *p) { memcpy(p, v_puw, (size_t)v_ny * 2 * sizeof(double)); }

/* Gauss-Lobatto points and integration weights from preprbl. */
void sref_grid(double *eta, double *wint) {
  memcpy(eta, v_eta, (size_t)v_nyp * sizeof(double));
  memcpy(wint, v_wint, (size_t)v_nyp * sizeof(double));
}

/* Plane statistics: nonlinbl calls boxamp at the first substep of a step
 * when iamp > 0 (bla/nonlinbl.f:425-432); amp(nyp,20) is copied out. */
void sref_set_iamp(int iamp) { v_iamp = iamp > 0 ? iamp : -1000000; }
void sref_get_amp(double *a) { memcpy(a, v_amp, (size_t)v_nyp * 20 * sizeof(double)); }

/* Pressure of the current state: the block of bla/bla.f:2486-2527 (nonlinp
 * on every xz-plane, linearp on every kz plane) with do_press set, as the
 * driver runs it after a step that saves a field.  Needs the variant built
 * with pressure = 1 (slot 8 holds p afterwards; linearp also recomputes
 * omega_x, omega_z in slots 4-5).  Returns -1 on a pressure = 0 build. */
int sref_pressure(double *re_part, double *im_part) {
  if (v_pressure != 1) return -1;
  if (v_spat) bla_ffun();
  v_do_press = 1;
  bla_press();
  v_do_press = 0;
  long n = slot_size();
  memcpy(re_part, v_ur + 7 * n, n * sizeof(double));
  memcpy(im_part, v_ui + 7 * n, n * sizeof(double));
  return 0;
}

/* xy statistics: the sampling block of bla/bla.f:2069-2107 (boxxys on every
 * xz-plane with weight dtn, then sumw(istat) += dtn) run on the current
 * state, as bla.f does at the start of a step that takes statistics.  With
 * reset != 0 xys and sumw are zeroed first (bla.f:1573 and the zeroed
 * allocation).  out receives xys(1:nx, 1:nyp, 1:nxys) of istat = 1 (x
 * fastest; the array's y extent is nyp/nproc+1), sumw_out sumw(1). */
void sref_xys(double dtn, int reset, double *out, double *sumw_out) {
  const long ly = (long)v_nyp / v_nproc + 1;
  if (reset) {
    memset(v_xys, 0, (size_t)v_nx * ly * v_nxys * v_mxys * sizeof(double));
    v_sumw[0] = 0.0;
  }
  const double dtn_saved = v_dtn;
  v_dtn = dtn;
  v_xysp = 1.0; /* istat = mod(int(t/xysp), mxys) + 1 = 1 */
  v_do_stat = 1;
  bla_xys();
  v_do_stat = 0;
  v_dtn = dtn_saved;
  for (long s = 0; s < v_nxys; ++s)
    for (long y = 0; y < v_nyp; ++y)
      memcpy(out + (s * v_nyp + y) * v_nx, v_xys + (s * ly + y) * v_nx, (size_t)v_nx * sizeof(double));
  *sumw_out = v_sumw[0];
}

/* LES as rparamles.f would leave it for an sgs.i with iles, cutoff_inv, iord,
 * chi, cs, ineg (bla/rparamles.f:31-60), ihighorder as given (the reference
 * default is 2), then the filter set-up of bla/bla.f:1489-1545 and
 * chi_scaled = chi/dstar (:2220).  Call after sref_setup, before sref_start.
 * iles = 2 (eddy viscosity, cs = 0 dynamic) needs an oracle built with
 * iiles_smag = 1. */
void sref_set_les(int iles, double cutoff_inv, int iord, double chi, int ihighorder, double cs, int ineg) {
  v_iles = iles; v_cutoff = 1.0 / cutoff_inv; v_iord = iord; v_chi = chi;
  v_ihighorder = ihighorder; v_cs = cs; v_ineg = ineg; v_prt = 0.6;
  v_chi_scaled = v_chi / v_dstar;
  bla_lesinit();
}

/* Filter tables: gewy1, gewy2, diags (nyp,5 each), gewspecx (nx/2+2),
 * gewspecz (nz/2+2), lpfxz (nx/2,nz). */
void sref_get_filter(double *g1, double *g2, double *dg, double *sx, double *sz, double *lpf) {
  memcpy(g1, v_gewy1, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(g2, v_gewy2, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(dg, v_diags, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(sx, v_gewspecx, (size_t)(v_nx / 2 + 2) * sizeof(double));
  memcpy(sz, v_gewspecz, (size_t)(v_nz / 2 + 2) * sizeof(double));
  memcpy(lpf, v_lpfxz, (size_t)(v_nx / 2) * v_nz * sizeof(double));
}

/* Secondary filter of the dynamic HPF model (bla/bla.f:1520-1545, after
 * sref_set_les with iles = 3, cs = 0): gewy12, gewy22, diags2 (nyp,5 each),
 * lpfxz2 and filtxz2 (nx/2,nz). */
void sref_get_filter2(double *g1, double *g2, double *dg, double *lpf, double *filt) {
  memcpy(g1, v_gewy12, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(g2, v_gewy22, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(dg, v_diags2, (size_t)v_nyp * 5 * sizeof(double));
  memcpy(lpf, v_lpfxz2, (size_t)(v_nx / 2) * v_nz * sizeof(double));
  memcpy(filt, v_filtxz2, (size_t)(v_nx / 2) * v_nz * sizeof(double));
}

/* High-pass filtered velocity gur,gui(memnx,memny,memnz,5), component 1..3. */
void sref_get_gu(int comp, double *re_part, double *im_part) {
  long n = slot_size();
  memcpy(re_part, v_gur + (long)(comp - 1) * n, n * sizeof(double));
  memcpy(im_part, v_gui + (long)(comp - 1) * n, n * sizeof(double));
}

/* SGS stress tau_ij (taur, taui slot 1..6: 11 12 13 22 23 33) of the last
 * les() call; its divergence sigma_i is in gur, gui slots 1..3. */
void sref_get_tau(int comp, double *re_part, double *im_part) {
  long n = slot_size();
  memcpy(re_part, v_taur + (long)(comp - 1) * n, n * sizeof(double));
  memcpy(im_part, v_taui + (long)(comp - 1) * n, n * sizeof(double));
}
