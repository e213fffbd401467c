// Device data layout of the resident spectral state.
//
// The reference keeps its main storage as two split real arrays
// ur/ui(memnx, memny, memnz, slot) (bla/par.f:111-120): kx fastest, then y,
// then kz.  On the device every field is interleaved complex and y-major:
//
//     field[y][kz][kx]          (double2, kx fastest)
//
// so an xz-plane (what step 2 transforms) is one contiguous nz*nx/2 block and
// a y-pencil (what step 3 solves) is a strided column whose neighbouring
// pencils sit in neighbouring addresses: both steps read fully coalesced
// without a transpose.  "p" below is the pencil index kz*(nx/2)+kx and NP the
// number of pencils; slot s occupies [s][y][p].
#pragma once

namespace sb {

struct Dims {
  int nx, ny, nz;   // spectral modes (par.f nx, ny, nz); ny is also nyp here
  int nx2;          // stored kx modes, nx/2
  int nyp;          // y collocation points
  int nxp, nzp;     // 3/2-rule dealiasing grid
  int NP;           // pencils per field, nz*nx2
  int zodd;         // oddball kz index nz/2 (skipped by step 3)
  // the part of the domain this context computes (a shard of a multi-GPU
  // run; the whole domain otherwise): step 2 on the xz-planes y0 <= y < y1,
  // step 3 on the pencils p0 <= p < p1 (a slab of kz planes)
  int y0, y1;
  int p0, p1;
};

// Fringe forcing of a spatial simulation (bla/fring.f without wave or streak
// forcing): H -= lambda(x) (u - U_b(x, y)) for the three components, in
// physical space after the products.  lam[nxp]: the fringe function at every
// x point (bla/ffun.f; zero outside the fringe, where the reference applies
// nothing); base[3][nyp][nxp]: the base flow u, v, w in physical space.
// lam == nullptr: no fringe.
struct Fringe {
  const double* lam;
  const double* base;
};

}  // namespace sb
