// internal.h -- declarations shared by the host files of libpdhcg_b200.
#pragma once

#include "../../include/pdhcg.h"
#include "../../include/pdhcg_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

int pdhcg_b200_cone_length(cone_type_t type, int v_dim);
qp_problem_t *pdhcg_b200_problem_clone(const qp_problem_t *p);
// trim a result of qcqp_to_socp_qp's extended problem to the original sizes (qcqp.cpp)
void pdhcg_b200_restore_qcqp_result(pdhcg_result_t *r, const qp_problem_t *orig);
int pdhcg_b200_cancel_requested(void);

#ifdef __cplusplus
}
#endif
