#ifndef CLI_COMMON_H
#define CLI_COMMON_H

#include "aco_api.h"

/*
 * CLI helpers with the reference's output contract
 * (src/common/cli_common.c:8-85): "Route i: c1 c2 ..." lines (depots
 * omitted), "Cost: %.3f" and "best cost: %.3f" (parsed by the reference's
 * runners, tools/bash/solve_cuda.sh:161).
 */

#include "solution.h"

#ifdef __cplusplus
extern "C" {
#endif

ACO_API int cli_parse_int_arg(const char *s, int *out);
ACO_API unsigned int cli_parse_uint_arg(const char *s, int *ok);
ACO_API void cli_print_solution_routes(const Solution *best, int K);
ACO_API void cli_print_solution_cost(double best_cost);
ACO_API int cli_validate_solution_or_report(const Solution *best, int n, int K,
                                    double best_cost);

#ifdef __cplusplus
}
#endif

#endif
