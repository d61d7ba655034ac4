#ifndef INSTANCE_PARSER_H
#define INSTANCE_PARSER_H

#include "aco_api.h"

/*
 * TSPLIB-style EUC_2D CVRP reader (reference: include/instance_parser.h,
 * src/common/instance_parser.c:226-388).
 */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int vehicles;
  int capacity;
} VrpInstanceMeta;

/*
 * Reference behaviour: loads n+1 float coordinates and VEHICLES/CAPACITY, and
 * rejects any customer demand other than 1 (instance_parser.c:157-166).
 * Returns 0 on success, 1 on error (message on stderr).
 */
ACO_API int vrp_load_tsplib_euc2d_coords(const char *path, int *n_out,
                                 float **coords_x_out, float **coords_y_out,
                                 VrpInstanceMeta *meta_out);

/*
 * Demand extension: same as above but returns the n+1 demands (demand[0] must
 * be 0, customers >= 1) in *demand_out (malloc'ed; caller frees).
 */
ACO_API int vrp_load_tsplib_euc2d_coords_demands(const char *path, int *n_out,
                                         float **coords_x_out,
                                         float **coords_y_out,
                                         int **demand_out,
                                         VrpInstanceMeta *meta_out);

#ifdef __cplusplus
}
#endif

#endif
