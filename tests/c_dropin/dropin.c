/* dropin.c -- the reference host's per-pixel loop after the drop-in patch, as C.
 *
 * Test infrastructure: compiled by tests/test_c_dropin.py with gcc against
 * include/pmilos.h and linked to libpmilos_b200.so, so the C ABI is exercised by a
 * C compiler rather than through ctypes.
 *
 *   dropin layout            print sizeof/offsetof of every struct the header
 *                            declares (no device calls), one "name value" per line
 *   dropin invert IN OUT     read a case (layout below), then do what the patched
 *                            milos.c does in place of its per-pixel loop
 *                            (milos.c:958-1009): the pixels live in one
 *                            allocation each (milos.c reads the cube with
 *                            forParallel = 0, utilsFits.c:229), so they are packed
 *                            into one [npix][4][nlambda] array and inverted by one
 *                            pm_invert_batch call; then the first n_single pixels
 *                            again through pm_lm_mils, the batch-of-one form that
 *                            keeps the loop (the lm_mils call of milos.c:998)
 *
 * IN (native endianness):  int32 nlambda, npix, nterms, precision, has_psf,
 *   n_single; float64 lambda0, quantum[6]; float64 lambda[nlambda];
 *   float64 psf[nlambda] (if has_psf); int32 fix[11]; float64 guess[11];
 *   float32 cube[npix][4][nlambda]
 * OUT: float64 models[npix][11]; float32 chisq[npix]; int32 iters[npix];
 *   float32 bestfit[npix][4][nlambda]; then per single pixel: int32 rc,
 *   float64 model[11], float32 spectra[4][nlambda], float32 chisq, int32 iter
 */
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pmilos.h"

#define FIELD(T, f) printf("offsetof %s.%s %zu\n", #T, #f, offsetof(T, f))
#define SIZE(T) printf("sizeof %s %zu\n", #T, sizeof(T))

static int layout(void) {
  SIZE(pm_model);
  FIELD(pm_model, eta0); FIELD(pm_model, B); FIELD(pm_model, vlos); FIELD(pm_model, dopp);
  FIELD(pm_model, aa); FIELD(pm_model, gm); FIELD(pm_model, az); FIELD(pm_model, S0);
  FIELD(pm_model, S1); FIELD(pm_model, mac); FIELD(pm_model, alfa);
  SIZE(pm_line);
  FIELD(pm_line, lambda0); FIELD(pm_line, n_pi); FIELD(pm_line, n_sig); FIELD(pm_line, nup);
  FIELD(pm_line, nub); FIELD(pm_line, nur); FIELD(pm_line, wep); FIELD(pm_line, web); FIELD(pm_line, wer);
  FIELD(pm_line, gl); FIELD(pm_line, gu); FIELD(pm_line, geff); FIELD(pm_line, fo);
  SIZE(pm_config);
  FIELD(pm_config, nlambda); FIELD(pm_config, lambda); FIELD(pm_config, psf); FIELD(pm_config, weight);
  FIELD(pm_config, noise); FIELD(pm_config, ilambda); FIELD(pm_config, toplim); FIELD(pm_config, miter);
  FIELD(pm_config, fix); FIELD(pm_config, nterms); FIELD(pm_config, logclambda); FIELD(pm_config, mu);
  FIELD(pm_config, classical_estimates); FIELD(pm_config, precision); FIELD(pm_config, solver);
  SIZE(pm_stats);
  FIELD(pm_stats, pixels); FIELD(pm_stats, iterations); FIELD(pm_stats, accepted);
  FIELD(pm_stats, eigen_fallbacks); FIELD(pm_stats, kernel_ms); FIELD(pm_stats, total_ms);
  FIELD(pm_stats, graph_replays);
  SIZE(pm_tuning);
  FIELD(pm_tuning, variant); FIELD(pm_tuning, staging_depth); FIELD(pm_tuning, warps_per_block);
  FIELD(pm_tuning, graphs);
  SIZE(pm_fits_cube);
  FIELD(pm_fits_cube, naxis); FIELD(pm_fits_cube, naxes); FIELD(pm_fits_cube, axis_row);
  FIELD(pm_fits_cube, axis_col); FIELD(pm_fits_cube, axis_lambda); FIELD(pm_fits_cube, axis_stokes);
  FIELD(pm_fits_cube, from_ctype); FIELD(pm_fits_cube, nrows); FIELD(pm_fits_cube, ncols);
  FIELD(pm_fits_cube, npix); FIELD(pm_fits_cube, nlambda); FIELD(pm_fits_cube, data_offset);
  FIELD(pm_fits_cube, data_bytes);
  SIZE(pm_server_config);
  FIELD(pm_server_config, hbm_budget_bytes); FIELD(pm_server_config, max_inflight);
  FIELD(pm_server_config, linger_ms);
  SIZE(pm_scan_info);
  FIELD(pm_scan_info, npix); FIELD(pm_scan_info, grid); FIELD(pm_scan_info, rc); FIELD(pm_scan_info, submit_ms);
  FIELD(pm_scan_info, admit_ms); FIELD(pm_scan_info, done_ms); FIELD(pm_scan_info, iterations);
  SIZE(pm_server_stats);
  FIELD(pm_server_stats, scans_done); FIELD(pm_server_stats, pixels_done); FIELD(pm_server_stats, kernel_launches);
  FIELD(pm_server_stats, latency_p50_ms); FIELD(pm_server_stats, latency_p99_ms);
  FIELD(pm_server_stats, latency_max_ms); FIELD(pm_server_stats, busy_ms); FIELD(pm_server_stats, arena_peak_bytes);
  FIELD(pm_server_stats, prepass_launches);
  printf("abi_version %d\n", pm_abi_version());
  return 0;
}

static void *read_all(FILE *f, size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (!p || fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "dropin: short input\n");
    exit(2);
  }
  return p;
}

#define CHECK(call)                                                              \
  do {                                                                           \
    int rc_ = (call);                                                            \
    if (rc_ < 0) {                                                               \
      fprintf(stderr, "dropin: %s -> %d: %s\n", #call, rc_, pm_last_error());    \
      exit(1);                                                                   \
    }                                                                            \
  } while (0)

static int invert(const char *in_path, const char *out_path) {
  FILE *f = fopen(in_path, "rb");
  if (!f) return fprintf(stderr, "dropin: cannot open %s\n", in_path), 2;
  int32_t *hdr = read_all(f, sizeof(int32_t) * 6);
  const int nl = hdr[0], npix = hdr[1], nterms = hdr[2], precision = hdr[3], has_psf = hdr[4], n_single = hdr[5];
  double *q = read_all(f, sizeof(double) * 7);  /* lambda0, SLOI, LLOI, JLOI, SUPI, LUPI, JUPI */
  double *lam = read_all(f, sizeof(double) * nl);
  double *psf = has_psf ? read_all(f, sizeof(double) * nl) : NULL;
  int32_t *fix = read_all(f, sizeof(int32_t) * 11);
  double *guess = read_all(f, sizeof(double) * 11);
  const size_t n4 = (size_t)4 * nl;
  /* the reference's milos.x holds one allocation per pixel (forParallel = 0) */
  float **pixels = malloc(sizeof(float *) * (size_t)npix);
  for (int p = 0; p < npix; p++) pixels[p] = read_all(f, sizeof(float) * n4);
  fclose(f);

  /* once per run, after create_cuantic and the PSF taps (milos.c:248-392) */
  pm_line line;
  CHECK(pm_line_from_quantum(q[0], q[1], q[2], q[3], q[4], q[5], q[6], &line));
  pm_config cfg;
  memset(&cfg, 0, sizeof cfg);
  cfg.nlambda = nl;
  cfg.lambda = lam;
  cfg.psf = psf;
  for (int i = 0; i < 4; i++) cfg.weight[i] = 1.0;
  cfg.noise = 1e-6;  /* 1 / (S/N = 1000)^2 */
  cfg.ilambda = 0.1;
  cfg.toplim = 1e-12;
  cfg.miter = 50;
  for (int i = 0; i < 11; i++) cfg.fix[i] = fix[i];
  cfg.nterms = nterms;
  cfg.logclambda = 0;
  cfg.mu = 1.0;
  cfg.classical_estimates = 1;
  cfg.precision = precision;
  cfg.solver = PM_SOLVE_DEFAULT;
  pm_ctx *ctx = NULL;
  CHECK(pm_ctx_create(&line, &cfg, NULL, &ctx));

  pm_model init;
  memcpy(&init, guess, sizeof init);  /* Init_Model and pm_model share their layout */

  /* the per-pixel loop of milos.c:958-1009 becomes: pack, one batched call */
  float *cube = malloc(sizeof(float) * (size_t)npix * n4);
  for (int p = 0; p < npix; p++) memcpy(cube + (size_t)p * n4, pixels[p], sizeof(float) * n4);
  pm_model *models = malloc(sizeof(pm_model) * (size_t)npix);
  float *chisq = malloc(sizeof(float) * (size_t)npix);
  int *iters = malloc(sizeof(int) * (size_t)npix);
  float *bestfit = malloc(sizeof(float) * (size_t)npix * n4);
  CHECK(pm_invert_batch(ctx, npix, cube, NULL, PM_SLIGHT_NONE, &init, models, chisq, iters, bestfit, NULL,
                        PM_MEM_HOST));

  FILE *o = fopen(out_path, "wb");
  if (!o) return fprintf(stderr, "dropin: cannot write %s\n", out_path), 2;
  fwrite(models, sizeof(pm_model), (size_t)npix, o);
  fwrite(chisq, sizeof(float), (size_t)npix, o);
  fwrite(iters, sizeof(int), (size_t)npix, o);
  fwrite(bestfit, sizeof(float), (size_t)npix * n4, o);

  /* hosts that keep the loop: lm_mils(...) -> pm_lm_mils(...), pixel by pixel */
  float *spectra = malloc(sizeof(float) * n4);
  for (int p = 0; p < n_single && p < npix; p++) {
    pm_model m = init;
    float chi = 0.0f;
    int iter = 0;
    int32_t rc = pm_lm_mils(ctx, pixels[p], &m, spectra, &chi, NULL, &iter);
    if (rc < -1) {
      fprintf(stderr, "dropin: pm_lm_mils -> %d: %s\n", rc, pm_last_error());
      return 1;
    }
    fwrite(&rc, sizeof rc, 1, o);
    fwrite(&m, sizeof m, 1, o);
    fwrite(spectra, sizeof(float), n4, o);
    fwrite(&chi, sizeof chi, 1, o);
    fwrite(&iter, sizeof iter, 1, o);
  }
  fclose(o);
  CHECK(pm_ctx_destroy(ctx));
  for (int p = 0; p < npix; p++) free(pixels[p]);
  free(pixels); free(cube); free(models); free(chisq); free(iters); free(bestfit); free(spectra);
  free(hdr); free(q); free(lam); free(psf); free(fix); free(guess);
  return 0;
}

int main(int argc, char **argv) {
  if (argc == 2 && !strcmp(argv[1], "layout")) return layout();
  if (argc == 4 && !strcmp(argv[1], "invert")) return invert(argv[2], argv[3]);
  fprintf(stderr, "usage: dropin layout | dropin invert IN OUT\n");
  return 2;
}
