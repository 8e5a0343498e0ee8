/*
 * fortran_abi_check.c -- calls the force subroutines the way MEGA's Fortran
 * does: construct_fint_gpu with CONSTRUCT_FINT's own 46 arguments
 * (FINT.F90:16-25), every one by reference, arrays column-major ((3,N)
 * xyz per node, (6,N) Voigt per node, (20,N) state, GSTACK_DSHP(3,NNZ)),
 * 1-based neighbour lists; then checks that it returns what the
 * short-list drop-in mega_construct_fint returns for the same call, bit for
 * bit, on a LINIT call and on a loaded one, and that the NSNI LINIT fills
 * GSTACK_DDSHP.  Built with plain gcc against include/mega_gpu.h and
 * libmega_gpu.so; exit status 0 when every check passes.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/mega_gpu.h"

static uint64_t rng = 88172645463325252ull;
static double urand(void) { /* xorshift64, uniform in [0, 1) */
  rng ^= rng << 13; rng ^= rng >> 7; rng ^= rng << 17;
  return (double)(rng >> 11) * (1.0 / 9007199254740992.0);
}

#define CHECK(cond, msg) do { if (!(cond)) { fprintf(stderr, "FAIL: %s\n", msg); return 1; } } while (0)

int main(void) {
  const int nx = 6, ny = 6, nz = 10;
  const double h = 1.0e-3;
  int32_t n = nx * ny * nz;
  double *coo = malloc(sizeof(double) * 3 * n), *win = malloc(sizeof(double) * 3 * n);
  double *vol = malloc(sizeof(double) * n), *sml = calloc(6 * (size_t)n, sizeof(double));
  double *props = calloc(30 * (size_t)n, sizeof(double));
  int32_t *mat = malloc(sizeof(int32_t) * n), *ebcn = calloc(n, sizeof(int32_t));
  int k = 0;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix, ++k) {
        coo[3 * k] = (ix + 0.1 * (urand() - 0.5)) * h;
        coo[3 * k + 1] = (iy + 0.1 * (urand() - 0.5)) * h;
        coo[3 * k + 2] = (iz + 0.1 * (urand() - 0.5)) * h;
        for (int d = 0; d < 3; ++d) win[3 * k + d] = 2.0 * h;
        for (int d = 0; d < 6; ++d) sml[6 * k + d] = 0.5 * h;
        vol[k] = h * h * h;
        mat[k] = 2;
        /* PROPS(1..6) = nu, E, rho, sigma_y, B, C; PROPS(28..30) = lambda, mu, lambda + 2 mu */
        double nu = 0.3, E = 200e9, lam = E * nu / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
        double* pr = props + 30 * (size_t)k;
        pr[0] = nu; pr[1] = E; pr[2] = 7800.0; pr[3] = 300e6; pr[4] = 0.5; pr[5] = 1.0;
        pr[27] = lam; pr[28] = mu; pr[29] = lam + 2 * mu;
        ebcn[k] = iz == 0;
      }
  double dist_max[3] = {0.0, 0.0, 0.0};
  int32_t *gn = malloc(sizeof(int32_t) * n), *gstart = malloc(sizeof(int32_t) * n);
  int32_t *ijk = malloc(sizeof(int32_t) * 3 * n), gmaxn = 0;
  int64_t cap = (int64_t)n * 200, nnz = 0;
  int32_t* gstack = malloc(sizeof(int32_t) * cap);
  int st = mega_bin_search(n, coo, win, sml, dist_max, 2, 0, gn, gstart, gstack, cap, &gmaxn, ijk, &nnz);
  CHECK(st == 0, "mega_bin_search");
  int32_t dim_nn = (int32_t)nnz;

  mega_params p;
  mega_params_default(&p);
  p.ql_len = 0.1 * h;
  CHECK(mega_fint_control(&p) == 0, "mega_fint_control");

  double *shp = calloc(nnz, sizeof(double)), *dshp = calloc(3 * nnz, sizeof(double));
  double *ddshp = calloc(6 * nnz, sizeof(double));
  double *shp2 = calloc(nnz, sizeof(double)), *dshp2 = calloc(3 * nnz, sizeof(double));
  double *state = calloc(20 * (size_t)n, sizeof(double)), *state2 = calloc(20 * (size_t)n, sizeof(double));
  double *stress = calloc(6 * (size_t)n, sizeof(double)), *stress2 = calloc(6 * (size_t)n, sizeof(double));
  double *strain = calloc(6 * (size_t)n, sizeof(double)), *strain2 = calloc(6 * (size_t)n, sizeof(double));
  double *hs = calloc(6 * (size_t)n, sizeof(double)), *ss = calloc(6 * (size_t)n, sizeof(double));
  double *dinc = calloc(3 * (size_t)n, sizeof(double)), *dtot = calloc(3 * (size_t)n, sizeof(double));
  double *fint = calloc(3 * (size_t)n, sizeof(double)), *fext = calloc(3 * (size_t)n, sizeof(double));
  double *fint2 = calloc(3 * (size_t)n, sizeof(double)), *fext2 = calloc(3 * (size_t)n, sizeof(double));
  double *wv = calloc(n, sizeof(double)), *wv2 = calloc(n, sizeof(double));
  double *seq = calloc(n, sizeof(double)), *seq2 = calloc(n, sizeof(double)), *cdist = calloc(n, sizeof(double));
  double *dx = calloc(6 * (size_t)n, sizeof(double)), *dy = calloc(6 * (size_t)n, sizeof(double));
  double *dz = calloc(6 * (size_t)n, sizeof(double)), *mom = calloc(n, sizeof(double));
  double *area = calloc(3 * (size_t)n, sizeof(double)), *smv = calloc(n, sizeof(double));
  double *fac = calloc(3 * (size_t)n, sizeof(double)), *bf = calloc(3 * (size_t)n, sizeof(double));
  double *ginvk = calloc(9 * (size_t)n, sizeof(double));
  int32_t *ghost = calloc(n, sizeof(int32_t)), *body = malloc(sizeof(int32_t) * n);
  for (int i = 0; i < n; ++i) body[i] = 1;
  double gw = 0.0, gw2 = 0.0, dlt_fint = -1.0, dlt = 1.0e-8;

  /* LINIT, DNI */
  int32_t linit = 1;
  p.itype_int = 0;
  CHECK(mega_fint_control(&p) == 0, "mega_fint_control");
  st = construct_fint_gpu(win, vol, &n, coo, coo, sml, area, smv, fac, ghost, props, state, stress, strain, hs, ss,
                          dinc, dtot, mat, ebcn, gn, gstart, &dim_nn, gstack, shp, dshp, ddshp, &gmaxn, ginvk, &linit,
                          fint, fext, &dlt_fint, cdist, wv, dx, dy, dz, mom, mom, mom, bf, &gw, body, seq, &dlt);
  CHECK(st == 0, "construct_fint_gpu LINIT");
  st = mega_construct_fint(&p, n, coo, win, vol, props, mat, ebcn, NULL, state2, stress2, strain2, dinc, dtot, gn,
                           gstart, gstack, nnz, shp2, dshp2, 1, dlt, fint2, fext2, wv2, seq2, &gw2);
  CHECK(st == 0, "mega_construct_fint LINIT");
  CHECK(memcmp(shp, shp2, sizeof(double) * nnz) == 0, "GSTACK_SHP differs");
  CHECK(memcmp(dshp, dshp2, sizeof(double) * 3 * nnz) == 0, "GSTACK_DSHP differs");
  CHECK(dlt_fint == -1.0, "DLT_FINT written");

  /* a loaded call: a smooth compression plus noise */
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      const double x = coo[3 * i + d];
      dtot[3 * i + d] = (d == 2 ? -0.02 : 0.006) * x + 1e-7 * (urand() - 0.5);
      dinc[3 * i + d] = 0.05 * dtot[3 * i + d];
    }
  linit = 0;
  st = construct_fint_gpu(win, vol, &n, coo, coo, sml, area, smv, fac, ghost, props, state, stress, strain, hs, ss,
                          dinc, dtot, mat, ebcn, gn, gstart, &dim_nn, gstack, shp, dshp, ddshp, &gmaxn, ginvk, &linit,
                          fint, fext, &dlt_fint, cdist, wv, dx, dy, dz, mom, mom, mom, bf, &gw, body, seq, &dlt);
  CHECK(st == 0, "construct_fint_gpu");
  st = mega_construct_fint(&p, n, coo, win, vol, props, mat, ebcn, NULL, state2, stress2, strain2, dinc, dtot, gn,
                           gstart, gstack, nnz, shp2, dshp2, 0, dlt, fint2, fext2, wv2, seq2, &gw2);
  CHECK(st == 0, "mega_construct_fint");
  CHECK(memcmp(fint, fint2, sizeof(double) * 3 * n) == 0, "FINT differs");
  CHECK(memcmp(stress, stress2, sizeof(double) * 6 * n) == 0, "GSTRESS differs");
  CHECK(memcmp(state, state2, sizeof(double) * 20 * n) == 0, "GSTATE differs");
  CHECK(gw == gw2, "GINT_WORK differs");
  double fmax = 0.0;
  for (int i = 0; i < 3 * n; ++i) fmax = fmax > fabs(fint[i]) ? fmax : fabs(fint[i]);
  CHECK(fmax > 0.0, "no internal force");

  /* NSNI LINIT: the second derivatives are written */
  p.itype_int = 2;
  CHECK(mega_fint_control(&p) == 0, "mega_fint_control NSNI");
  linit = 1;
  memset(stress, 0, sizeof(double) * 6 * n);
  memset(dinc, 0, sizeof(double) * 3 * n);
  memset(dtot, 0, sizeof(double) * 3 * n);
  st = construct_fint_gpu(win, vol, &n, coo, coo, sml, area, smv, fac, ghost, props, state, stress, strain, hs, ss,
                          dinc, dtot, mat, ebcn, gn, gstart, &dim_nn, gstack, shp, dshp, ddshp, &gmaxn, ginvk, &linit,
                          fint, fext, &dlt_fint, cdist, wv, dx, dy, dz, mom, mom, mom, bf, &gw, body, seq, &dlt);
  CHECK(st == 0, "construct_fint_gpu NSNI LINIT");
  double dmax = 0.0;
  for (int64_t q = 0; q < 6 * nnz; ++q) dmax = dmax > fabs(ddshp[q]) ? dmax : fabs(ddshp[q]);
  CHECK(dmax > 0.0, "GSTACK_DDSHP not written");
  printf("OK n=%d nnz=%lld\n", (int)n, (long long)nnz);
  return 0;
}
