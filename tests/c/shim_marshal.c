/* shim_marshal.c -- the Fortran shim's marshalling (fortran/bmadgpu_mod.f90, track_on_gpu),
 * restated in C, through the C-ABI: coord_struct-like records are gathered into the column-major
 * vec(n,6) buffer the shim allocates (element (j,i) at offset (i-1)*n + (j-1), which is the SoA
 * layout vec[i*n + j] of bmadgpu_bunch), tracked with bmadgpu_track_bunch for n_turns starting at
 * turn0, and scattered back with the shim's bookkeeping: lost particles get ix_ele (1-based),
 * ix_turn and location; survivors get ix_ele = ix_end and location downstream_end.
 *
 * usage: shim_marshal <elements.bin> <param.bin> <records.bin> <n> <ix_start> <ix_end> <turn0> <n_turns> <out.bin>
 * records: n x struct rec (below), read and written back. Exit status 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bmadgpu.h"

struct rec {                  /* the coord_struct fields the shim moves */
  double vec[6], beta, t;
  int32_t state, ix_ele, ix_turn, location;
};

static void* slurp(const char* path, size_t* size) {
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  void* p = malloc((size_t)n);
  if (p && fread(p, 1, (size_t)n, f) != (size_t)n) { free(p); p = NULL; }
  fclose(f);
  *size = (size_t)n;
  return p;
}

int main(int argc, char** argv) {
  if (argc != 10) return 2;
  size_t ne_bytes, np_bytes, nr_bytes;
  bmadgpu_element* eles = (bmadgpu_element*)slurp(argv[1], &ne_bytes);
  bmadgpu_param* param = (bmadgpu_param*)slurp(argv[2], &np_bytes);
  struct rec* r = (struct rec*)slurp(argv[3], &nr_bytes);
  const int64_t n = atoll(argv[4]);
  const int32_t ix_start = atoi(argv[5]), ix_end = atoi(argv[6]), turn0 = atoi(argv[7]), n_turns = atoi(argv[8]);
  if (!eles || !param || !r || nr_bytes != (size_t)n * sizeof(struct rec) || np_bytes != sizeof(bmadgpu_param)) return 3;
  const int32_t n_ele = (int32_t)(ne_bytes / sizeof(bmadgpu_element));

  bmadgpu_ctx* ctx = NULL;
  bmadgpu_lattice* lat = NULL;
  if (bmadgpu_ctx_create(0, &ctx) || bmadgpu_lattice_create(ctx, eles, n_ele, param, &lat)) {
    fprintf(stderr, "%s\n", bmadgpu_last_error());
    return 4;
  }
  /* allocate (vec(n, 6), beta(n), t(n), state(n), ix_ele(n), ix_turn(n), location(n)) */
  double* vec = malloc(sizeof(double) * 6 * n);
  double* beta = malloc(sizeof(double) * n);
  double* t = malloc(sizeof(double) * n);
  int32_t* state = malloc(sizeof(int32_t) * n);
  int32_t* ix_ele = malloc(sizeof(int32_t) * n);
  int32_t* ix_turn = malloc(sizeof(int32_t) * n);
  int32_t* location = malloc(sizeof(int32_t) * n);
  for (int64_t j = 1; j <= n; j++) {
    for (int i = 1; i <= 6; i++) vec[(i - 1) * n + (j - 1)] = r[j - 1].vec[i - 1];   /* vec(j, i) */
    beta[j - 1] = r[j - 1].beta;
    t[j - 1] = r[j - 1].t;
    state[j - 1] = r[j - 1].state;
    ix_ele[j - 1] = -1;
    ix_turn[j - 1] = -1;
    location[j - 1] = 0;
  }
  bmadgpu_bunch b = {n, vec, beta, t, state, ix_ele, ix_turn, location};
  if (bmadgpu_track_bunch(ctx, lat, &b, ix_start, ix_end, turn0, n_turns, NULL)) {
    fprintf(stderr, "%s\n", bmadgpu_last_error());
    return 5;
  }
  for (int64_t j = 1; j <= n; j++) {
    struct rec* p = &r[j - 1];
    for (int i = 1; i <= 6; i++) p->vec[i - 1] = vec[(i - 1) * n + (j - 1)];
    p->beta = beta[j - 1];
    p->t = t[j - 1];
    p->state = state[j - 1];
    if (ix_ele[j - 1] >= 0) {          /* lost in this call */
      p->ix_ele = ix_ele[j - 1] + 1;
      p->ix_turn = ix_turn[j - 1];
      p->location = location[j - 1];
    } else if (state[j - 1] == BMADGPU_ALIVE) {
      p->ix_ele = ix_end;
      p->location = BMADGPU_DOWNSTREAM_END;
    }
  }
  FILE* f = fopen(argv[9], "wb");
  if (!f || fwrite(r, sizeof(struct rec), (size_t)n, f) != (size_t)n) return 6;
  fclose(f);
  bmadgpu_lattice_destroy(lat);
  bmadgpu_ctx_destroy(ctx);
  return 0;
}
