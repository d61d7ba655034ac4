/*
 * TSPLIB EUC_2D CVRP reader.  Accepts the same header keys and section layout
 * as the reference (src/common/instance_parser.c:226-388): DIMENSION (n+1),
 * VEHICLES, CAPACITY ("KEY: v", "KEY : v" or "KEY v"), NODE_COORD_SECTION
 * ("id x y" for n+1 nodes, depot first) and DEMAND_SECTION ("id d").
 * An optional DEPOT_SECTION ("1", "-1") may only name node 1.
 * Missing VEHICLES/CAPACITY/DEMAND_SECTION, a nonzero depot demand or a
 * non-positive capacity are errors, as in the reference.
 *
 * vrp_load_tsplib_euc2d_coords keeps the reference's unit-demand rule;
 * vrp_load_tsplib_euc2d_coords_demands accepts any customer demand >= 1.
 */
#include "instance_parser.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int header_int(const char *line, size_t keylen, int *out) {
  const char *p = line + keylen;
  while (*p == ' ' || *p == '\t' || *p == ':') ++p;
  char *end = NULL;
  long v = strtol(p, &end, 10);
  if (end == p) return 0;
  *out = (int)v;
  return 1;
}

static int load(const char *path, int *n_out, float **xo, float **yo,
                int **demand_out, VrpInstanceMeta *meta_out, int unit_only) {
  FILE *f = fopen(path, "r");
  if (!f) {
    perror("fopen");
    return 1;
  }
  int n = 0, K = 0, cap = 0;
  int have_coords = 0, have_demands = 0;
  float *x = NULL, *y = NULL;
  int *d = NULL;
  char line[512];
  int err = 0;
  while (!err && fgets(line, sizeof(line), f)) {
    if (strncmp(line, "DIMENSION", 9) == 0) {
      int dim = 0;
      if (header_int(line, 9, &dim)) n = dim - 1;
    } else if (strncmp(line, "VEHICLES", 8) == 0) {
      header_int(line, 8, &K);
    } else if (strncmp(line, "CAPACITY", 8) == 0) {
      header_int(line, 8, &cap);
    } else if (strncmp(line, "NODE_COORD_SECTION", 18) == 0) {
      if (n <= 0) {
        fprintf(stderr, "DIMENSION must be defined before NODE_COORD_SECTION\n");
        err = 1;
        break;
      }
      free(x);
      free(y);
      x = (float *)malloc(sizeof(float) * ((size_t)n + 1));
      y = (float *)malloc(sizeof(float) * ((size_t)n + 1));
      if (!x || !y) { err = 1; break; }
      for (int i = 0; i <= n; ++i) {
        int id;
        double cx, cy;
        if (fscanf(f, "%d %lf %lf", &id, &cx, &cy) != 3) {
          fprintf(stderr, "Failed to read coordinates at index %d\n", i);
          err = 1;
          break;
        }
        x[i] = (float)cx;
        y[i] = (float)cy;
      }
      have_coords = !err;
    } else if (strncmp(line, "DEMAND_SECTION", 14) == 0) {
      if (n <= 0) {
        fprintf(stderr, "DIMENSION must be defined before DEMAND_SECTION\n");
        err = 1;
        break;
      }
      free(d);
      d = (int *)malloc(sizeof(int) * ((size_t)n + 1));
      if (!d) { err = 1; break; }
      for (int i = 0; i <= n; ++i) {
        int id;
        if (fscanf(f, "%d %d", &id, &d[i]) != 2) {
          fprintf(stderr, "Failed to read demands at index %d\n", i);
          err = 1;
          break;
        }
      }
      have_demands = !err;
    } else if (strncmp(line, "DEPOT_SECTION", 13) == 0) {
      /* Depot ids up to -1: node 1 (index 0) must be the only depot, the
       * layout every solver here and in the reference assumes. */
      int id = 0, count = 0;
      while (fscanf(f, "%d", &id) == 1 && id != -1) {
        if (id != 1 || ++count > 1) {
          fprintf(stderr, "Only node 1 may be the depot (DEPOT_SECTION) in %s\n", path);
          err = 1;
          break;
        }
      }
    }
  }
  fclose(f);
  if (!err && (n <= 0 || !have_coords)) {
    fprintf(stderr, "Invalid or missing DIMENSION/NODE_COORD_SECTION\n");
    err = 1;
  }
  if (!err && (K <= 0 || cap <= 0 || !have_demands)) {
    if (K <= 0 || !have_demands || cap == 0) {
      fprintf(stderr, "Missing VEHICLES/CAPACITY/DEMAND_SECTION in %s\n", path);
    } else {
      fprintf(stderr, "CAPACITY must be positive in %s\n", path);
    }
    err = 1;
  }
  if (!err && d[0] != 0) {
    fprintf(stderr, "Depot demand must be 0 in %s\n", path);
    err = 1;
  }
  for (int i = 1; !err && i <= n; ++i) {
    if (unit_only && d[i] != 1) {
      fprintf(stderr, "Customer demand must be 1 for all customers in %s\n", path);
      err = 1;
    } else if (d[i] < 1) {
      fprintf(stderr, "Customer demand must be >= 1 in %s\n", path);
      err = 1;
    }
  }
  if (err) {
    free(x);
    free(y);
    free(d);
    return 1;
  }
  *n_out = n;
  *xo = x;
  *yo = y;
  if (demand_out) *demand_out = d; else free(d);
  if (meta_out) {
    meta_out->vehicles = K;
    meta_out->capacity = cap;
  }
  return 0;
}

int vrp_load_tsplib_euc2d_coords(const char *path, int *n_out,
                                 float **coords_x_out, float **coords_y_out,
                                 VrpInstanceMeta *meta_out) {
  return load(path, n_out, coords_x_out, coords_y_out, NULL, meta_out, 1);
}

int vrp_load_tsplib_euc2d_coords_demands(const char *path, int *n_out,
                                         float **coords_x_out,
                                         float **coords_y_out,
                                         int **demand_out,
                                         VrpInstanceMeta *meta_out) {
  return load(path, n_out, coords_x_out, coords_y_out, demand_out, meta_out, 0);
}
