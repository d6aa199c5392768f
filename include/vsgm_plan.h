/* Plain-old-data plan tables shared by the planner, the CUDA engine, the C ABI
 * and the CPU oracle.  One vsgm_plan is the flattened form of the reference's
 * Plan + DevPlan pair (src/query/plan.h:61-580, src/query/dev_plan.h:128-313):
 * the execution sequence, the per-level vertex groups and the per-vertex
 * connectivity / condition tables, all indexed by pattern vertex id. */
#ifndef VSGM_PLAN_TYPES_H
#define VSGM_PLAN_TYPES_H

#include <stdint.h>

#define VSGM_MAX_QV 7   /* kMaxQueryVerticesNum, src/common/meta.h:37 */
#define VSGM_MAX_OPS 24 /* longest exec sequence of a 7-vertex pattern is 16 */

/* Operation codes keep TraversalOperation's numbering (src/query/plan.h:14-21). */
enum vsgm_op_type {
  VSGM_COMPUTE = 0,
  VSGM_COMPUTE_PATH_COUNT = 1,
  VSGM_MATERIALIZE = 2,
  VSGM_FILTER_COMPUTE = 3,
  VSGM_COUNT = 4,
  VSGM_COMPUTE_COUNT = 5
};

/* Condition operators keep CondOperator's numbering (src/common/meta.h:39). */
enum vsgm_cond_op { VSGM_LESS_THAN = 0, VSGM_LARGER_THAN = 1, VSGM_NON_EQUAL = 2, VSGM_OPERATOR_NONE = 3 };

/* A group of pattern vertices (DevConnType, src/query/dev_plan.h:10-60). */
typedef struct vsgm_vgroup {
  uint8_t count;
  uint8_t v[VSGM_MAX_QV];
} vsgm_vgroup;

/* A list of (operator, operand) conditions (DevCondArrayType, src/query/dev_plan.h:62-113).
 * Condition i reads: candidate  op[i]  M[v[i]]. */
typedef struct vsgm_conds {
  uint8_t count;
  uint8_t op[VSGM_MAX_QV];
  uint8_t v[VSGM_MAX_QV];
} vsgm_conds;

typedef struct vsgm_plan {
  uint32_t n_vertices;  /* pattern vertices (<= 7) */
  uint32_t n_edges;     /* undirected pattern edges */
  int32_t hop;          /* Plan::GetHop: halo depth a view needs */
  uint32_t root_degree; /* Plan::GetRootDegree */
  uint32_t root;        /* first vertex of the search sequence */
  uint32_t n_ops;       /* length of the execution sequence */
  uint8_t adj[VSGM_MAX_QV];               /* bit j of adj[i] <=> pattern edge (i, j) */
  uint8_t order[VSGM_MAX_QV][VSGM_MAX_QV]; /* GetConditionType(i, j) of the query */
  uint8_t seq[VSGM_MAX_QV];               /* search sequence */
  uint8_t op_type[VSGM_MAX_OPS];
  uint8_t op_vertex[VSGM_MAX_OPS]; /* COUNT carries n_vertices, as in the reference */
  vsgm_vgroup backward[VSGM_MAX_QV];       /* backward connectivity per vertex */
  vsgm_conds compute_cond[VSGM_MAX_QV];    /* GetComputeCondition */
  vsgm_conds materialize_cond[VSGM_MAX_QV]; /* GetMaterializeCondition */
  vsgm_conds filter_cond[VSGM_MAX_QV];     /* GetFilterCondition */
  vsgm_vgroup materialized[VSGM_MAX_OPS];   /* materialized vertices before op i */
  vsgm_vgroup computed_unmat[VSGM_MAX_OPS]; /* computed, unmaterialized vertices before op i */
} vsgm_plan;

#endif
