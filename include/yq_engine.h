/*
 * yq_engine.h — C entry to the C++ operator layer (libyq_engine.so).
 *
 * The operator layer mirrors YallaSQL's pull-based physical operators
 * (`YallaSQL::Operator::init()` / `BatchID next(CacheManager&)`,
 * include/engine/operators/operator.hpp:12-60) over columnar batches with one
 * null byte per row (include/batch.hpp:21-145) and a cache manager with a
 * device-memory budget (include/engine/cache_manager.hpp:11-88). Operators call
 * the kernels through include/yq_ops.h only. The reference builds the operator
 * tree from DuckDB's logical plan (src/engine/operators/operator.cpp:14-44);
 * DuckDB is not part of this path, so a host assembles the same tree here
 * node by node, with expressions already compiled to yq_program form.
 *
 * Input columns live in HOST memory; the scan streams them to the device as
 * 4 MB batches (include/config.hpp:28-36 sizing) through two pinned staging
 * buffers and a copy stream, so the copy of batch k+1 overlaps the kernels of
 * batch k (GetOperator::storeBuffer copies synchronously,
 * src/engine/operators/get_operator.cpp:125-148). Results come back to host
 * memory owned by the result object.
 */
#ifndef YQ_ENGINE_H
#define YQ_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#include "yq_ops.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct yq_plan yq_plan;
typedef struct yq_result yq_result;

/* A host column: `rows` values of `width` bytes at `data`, nulls one byte per
 * row or NULL. Pinned host memory is copied directly; pageable memory is
 * staged through the scan's pinned buffers. */
typedef struct yq_host_column {
  const void* data;
  const uint8_t* nulls;
  int32_t type;
  int32_t width;
} yq_host_column;

/* A plan owns its operators, a compute stream, a copy stream and a cache
 * manager whose device budget is `gpu_budget_bytes` (0 = 1 GiB, the
 * reference's MAX_LIMIT_GPU_CACHE, include/config.hpp:19). Batches beyond the
 * budget move to pinned host memory and come back on demand. */
yq_plan* yq_plan_create(uint64_t gpu_budget_bytes);
/* The host tier's budget and the directory of the file tier (the reference's
 * MAX_LIMIT_CPU_CACHE and cacheDir, include/config.hpp:17 and
 * CacheManager::handleOverflow(Device::CPU),
 * include/engine/cache_manager.hpp:82-85). When the batches spilled to pinned
 * host memory exceed `host_budget_bytes`, the oldest move to files in
 * `cache_dir`, written by a background task, null bytes included; they are
 * read back (and the file removed) when an operator asks for them. 0 (the
 * default) keeps spilled batches in host memory without limit. Returns
 * YQ_ERR_INVALID_ARG for a budget without a directory. */
int yq_plan_set_spill(yq_plan* plan, uint64_t host_budget_bytes, const char* cache_dir);
void yq_plan_destroy(yq_plan* plan);
/* Node builders return the new node id (>= 0) or -yq_status. */
int yq_plan_scan(yq_plan* plan, const yq_host_column* cols, int32_t ncols, uint64_t rows,
                 uint32_t batch_rows /* 0 = 4 MB batches */);
/* A table read from CSV text, GetOperator's place in the tree
 * (src/engine/operators/get_operator.cpp:17-109): `text` (host, nbytes) is
 * the file after its header line; field_types[f] is CSV field f's type (the
 * header-tag rule of Table::inferDBSchema); `project` lists the fields to
 * keep, in output order; text columns get `text_width`-byte slots. The text
 * goes to the device once and is converted batch by batch (yq_csv_index,
 * yq_csv_parse). Must stay valid until the plan executes. */
int yq_plan_scan_csv(yq_plan* plan, const uint8_t* text, uint64_t nbytes, const int32_t* field_types,
                     int32_t nfields, const int32_t* project, int32_t nproj, int32_t text_width,
                     uint32_t batch_rows /* 0 = 4 MB batches */);
int yq_plan_filter(yq_plan* plan, int32_t child, const yq_program* predicate,
                   const yq_constants* constants);
int yq_plan_project(yq_plan* plan, int32_t child, const yq_projection* proj, int32_t nproj,
                    const yq_constants* constants);
int yq_plan_aggregate(yq_plan* plan, int32_t child, const yq_agg_spec* aggs, int32_t nagg,
                      const yq_constants* constants);
int yq_plan_order(yq_plan* plan, int32_t child, int32_t key_col, int32_t descending,
                  int32_t nulls_first);
/* ORDER BY several keys, most significant first (the reference sorts by
 * `orders[0]` only, include/engine/operators/order_operator.hpp:277). One key
 * takes the out-of-core merge path (yq_order_by); several keys, or a text key
 * longer than 32 significant bytes, sort the whole input at once
 * (yq_sort_indices_multi) and gather. */
int yq_plan_order_multi(yq_plan* plan, int32_t child, const int32_t* keys, const int32_t* descending,
                        const int32_t* nulls_first, int32_t nkeys);
/* SELECT key, aggregates GROUP BY key (the reference's AggregateOperator
 * ignores the groups, include/engine/operators/aggregate_operator.hpp:84-104):
 * one output row per distinct key, ascending, NULL group last; columns = the
 * key, then one per aggregate with yq_group_by's types (COUNT INT64, SUM of
 * integers INT64, SUM of floats and AVG FLOAT64, MIN/MAX the input type). */
int yq_plan_group_by(yq_plan* plan, int32_t child, int32_t key_col, const yq_group_agg* aggs, int32_t nagg);
int yq_plan_join(yq_plan* plan, int32_t left, int32_t right, const yq_join_cond* conds,
                 int32_t ncond);
/* A join whose condition is an OR of ANDs: conds[i] belongs to disjunct group
 * disjunct[i] (yq_join_project_or). The reference throws on OR in a join
 * condition (include/engine/operators/expressions/filters/conjunction_join.hpp:113-114). */
int yq_plan_join_or(yq_plan* plan, int32_t left, int32_t right, const yq_join_cond* conds,
                    const int32_t* disjunct, int32_t ncond);
int yq_plan_cross(yq_plan* plan, int32_t left, int32_t right);

/* Pull every batch from `root` (ExecutorEngine::execute's loop,
 * src/engine/executor_engine.cpp:28-38), copy the result to host memory and
 * return it in *out (free with yq_result_destroy). */
int yq_plan_execute(yq_plan* plan, int32_t root, yq_result** out);

uint64_t yq_result_rows(const yq_result* r);
int32_t yq_result_ncols(const yq_result* r);
/* Host view of result column c (valid until yq_result_destroy). */
int yq_result_column(const yq_result* r, int32_t c, yq_host_column* out);
void yq_result_destroy(yq_result* r);

/* Statistics of the last execute: batches pulled, bytes copied host->device
 * and device->host, device milliseconds of the compute stream, and the moves
 * of the cache manager's spill tiers. */
typedef struct yq_plan_stats {
  uint64_t batches;
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  double compute_ms;
  uint64_t spilled_batches; /* device -> pinned host moves */
  uint64_t disk_batches;    /* pinned host -> file moves */
} yq_plan_stats;
int yq_plan_stats_read(const yq_plan* plan, yq_plan_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* YQ_ENGINE_H */
