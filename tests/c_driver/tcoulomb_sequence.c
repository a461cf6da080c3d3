/*
 * tcoulomb_sequence.c -- a plain C caller of the library, built against
 * include/ewald_b200.h alone (no Python, no ctypes), that replays the order in
 * which DFTB+'s SCC loop drives TCoulomb (src/dftbp/dftb/hamiltonian.F90:229-233
 * and the gradient and stress calls after convergence):
 *
 *   updateLatVecs -> updateCoords -> { updateCharges -> updateShifts } x nscc
 *   -> addGradients (shift and force) -> addStress (stock invRStress, and the
 *   NFFT-based stress) ; then one ewald_potential_force on the library surface.
 *
 * Usage: tcoulomb_sequence <in.bin> <out.bin>
 *   in.bin : int32 n, int32 nscc, double tol, double tol_ewald,
 *            double lat_cols[9], double coords[3n] (atom-major),
 *            double dq[nscc][n]
 *   out.bin: double shift[nscc][n], double shift_f[n], double force[3n],
 *            double sigma_stock[9], double sigma_fast[9],
 *            double pot_lib[n], double force_lib[3n]
 * Exit status: 0, or the first non-zero library status (its message on stderr).
 */
#include <stdio.h>
#include <stdlib.h>

#include "ewald_b200.h"

static int check(int rc, const char* where) {
  if (rc != EWG_OK) fprintf(stderr, "%s: %s (status %d)\n", where, ewg_status_string(rc), rc);
  return rc;
}

static int read_all(FILE* f, void* p, size_t size, size_t count) {
  return fread(p, size, count, f) == count ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) return 2;
  int n = 0, nscc = 0;
  double tol = 0.0, tol_ewald = 0.0, lat_cols[9];
  if (read_all(in, &n, sizeof(int), 1) || read_all(in, &nscc, sizeof(int), 1) ||
      read_all(in, &tol, sizeof(double), 1) || read_all(in, &tol_ewald, sizeof(double), 1) ||
      read_all(in, lat_cols, sizeof(double), 9) || n <= 0 || nscc <= 0) {
    fclose(in);
    return 2;
  }
  double* coords = malloc(sizeof(double) * 3 * (size_t)n);
  double* dq = malloc(sizeof(double) * (size_t)nscc * n);
  double* shift = malloc(sizeof(double) * (size_t)nscc * n);
  double* shift_f = malloc(sizeof(double) * (size_t)n);
  double* force = malloc(sizeof(double) * 3 * (size_t)n);
  double* positions = malloc(sizeof(double) * 3 * (size_t)n);
  double* pot_lib = malloc(sizeof(double) * (size_t)n);
  double* force_lib = malloc(sizeof(double) * 3 * (size_t)n);
  double sigma_stock[9], sigma_fast[9], lat_rows[9];
  int bad = read_all(in, coords, sizeof(double), 3 * (size_t)n) ||
            read_all(in, dq, sizeof(double), (size_t)nscc * n);
  fclose(in);
  if (bad) return 2;

  ewg_context* ctx = NULL;
  int rc = check(ewg_create(&ctx, 0, EWG_PRECISION_FP64), "ewg_create");
  if (!rc) rc = check(ewg_set_lattice(ctx, lat_cols), "ewg_set_lattice");
  if (!rc) rc = check(ewg_set_coords(ctx, n, coords), "ewg_set_coords");
  for (int k = 0; k < nscc && !rc; ++k) {
    rc = check(ewg_set_charges(ctx, dq + (size_t)k * n), "ewg_set_charges");
    if (!rc) rc = check(ewg_shift(ctx, tol, shift + (size_t)k * n), "ewg_shift");
  }
  if (!rc) rc = check(ewg_shift_force(ctx, tol, shift_f, force), "ewg_shift_force");
  if (!rc) rc = check(ewg_stress(ctx, tol_ewald, 0.0, sigma_stock), "ewg_stress");
  if (!rc) rc = check(ewg_stress_fast(ctx, tol, sigma_fast), "ewg_stress_fast");
  /* The library surface: positions(N,3) and lattice rows, Fortran layouts. */
  for (int i = 0; i < n && !rc; ++i)
    for (int d = 0; d < 3; ++d) positions[i + (size_t)n * d] = coords[d + 3 * (size_t)i];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) lat_rows[i + 3 * d] = lat_cols[d + 3 * i];
  if (!rc)
    rc = check(ewg_potential_force(ctx, n, positions, dq + (size_t)(nscc - 1) * n, lat_rows, tol,
                                   pot_lib, force_lib, NULL),
               "ewg_potential_force");
  if (ctx) ewg_destroy(ctx);
  if (!rc) {
    FILE* out = fopen(argv[2], "wb");
    if (!out) return 2;
    fwrite(shift, sizeof(double), (size_t)nscc * n, out);
    fwrite(shift_f, sizeof(double), (size_t)n, out);
    fwrite(force, sizeof(double), 3 * (size_t)n, out);
    fwrite(sigma_stock, sizeof(double), 9, out);
    fwrite(sigma_fast, sizeof(double), 9, out);
    fwrite(pot_lib, sizeof(double), (size_t)n, out);
    fwrite(force_lib, sizeof(double), 3 * (size_t)n, out);
    fclose(out);
  }
  free(coords);
  free(dq);
  free(shift);
  free(shift_f);
  free(force);
  free(positions);
  free(pot_lib);
  free(force_lib);
  return rc;
}
