/* oracle.h — C API of the f64 CPU oracle (a restatement of the reference's exact
 * evaluator and brick bake). TEST INFRASTRUCTURE ONLY: the tests, smoke() and the
 * CPU-baseline leg of bench.py call it as the checker; the product never does. */
#ifndef ICAM_ORACLE_H
#define ICAM_ORACLE_H

#include <stdint.h>

#include "../include/icam_solid.h"

#define ORACLE_AIR 0xffffffffu
#define ORACLE_SOLID 0xfffffffeu
#define ORACLE_READ 0xfffffff0u

#ifdef __cplusplus
extern "C" {
#endif

void* oracle_new(const IcamSolidDesc* d, char* err, int errlen);
void oracle_free(void* h);
void oracle_bbox(void* h, double* lo, double* hi);
int oracle_counts(void* h, int* nf, int* ne, int* nv);
void oracle_sdf(void* h, const double* pts, int64_t n, double bound, double* d_out, double* q_out,
                int32_t* kind_out, int32_t* id_out, uint8_t* unsure_out, int32_t* pops_out, int threads);
int oracle_candidates(void* h, const double* c, double r, double d, int32_t* out, int cap, int32_t* kinds);
int64_t oracle_decide(void* h, double hcell, const double* lo, const int64_t* nb, double clamp, const double* origin,
                      int threads, uint32_t* map, int64_t* read_idx, double* read_d, int64_t cap);
int64_t oracle_decide_rule(void* h, double hcell, const double* lo, const int64_t* nb, double clamp,
                           const double* origin, int threads, int tight, uint32_t* map, int64_t* read_idx,
                           double* read_d, int64_t cap);
void oracle_bricks(void* h, const double* firsts, int64_t n, double hcell, double clamp, int threads, double* f_out,
                   int16_t* q_out, int32_t* kind_out, uint32_t* words_out);

#ifdef __cplusplus
}
#endif

#endif
