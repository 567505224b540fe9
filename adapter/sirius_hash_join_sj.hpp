// Sirius-side glue for the sm_100a equi-join: what `sirius_physical_hash_join::execute`
// (src/op/sirius_physical_hash_join.cpp:1527-1955) calls instead of cuDF for its equi-joins
// (INNER, LEFT, SEMI, ANTI, MARK, FULL on 1..4 INT32/INT64 key columns).
//
// It maps cudf::column_view to sj_column, wraps the task's RMM resource as an sj_alloc (so the
// join's device memory is charged to the task's cuCascade reservation,
// src/pipeline/gpu_pipeline_task.cpp:523-525), and turns sj_status into the exceptions the
// operator's callers already handle: SJ_ERR_OOM -> rmm::out_of_memory (the OOM reschedule path,
// src/pipeline/gpu_pipeline_task.cpp:386-437), anything else -> std::runtime_error.
#pragma once

#include <memory>
#include <stdexcept>
#include <vector>

#include "cudf/column/column.hpp"
#include "cudf/table/table.hpp"
#include "cudf/table/table_view.hpp"
#include "rmm/cuda_stream_view.hpp"
#include "rmm/resource_ref.hpp"
#include "sj/sj_join.h"

namespace sirius::op::sj_adapter {

/// sj_type of a fixed-width cuDF type (DATE / TIMESTAMP / DURATION are stored as INT32 / INT64).
sj_type to_sj_type(cudf::data_type t);

/// Read-only view of a column: data at row 0, the null mask with the view's bit offset.
sj_column to_sj(cudf::column_view const& c);

/// The equi-key columns of a join condition as sj_columns (1..4; several form a composite key).
std::vector<sj_column> key_columns(cudf::table_view const& keys);

/// Throws rmm::out_of_memory for SJ_ERR_OOM, std::runtime_error otherwise (no-op for SJ_OK).
void check(sj_status st, char const* where);

/// The context of an sj_alloc over an RMM resource. libsj keeps the sj_alloc a table was built with
/// and frees the table's memory through it in sj_table_destroy, so a context handed to sj_build_ex
/// must live as long as the table: sj_hash_table holds it as a member.
struct rmm_alloc_ctx {
  rmm::device_async_resource_ref mr;
};

/// The built table of one BUILD_PROBE partition slot: replaces cudf::hash_join /
/// cudf::distinct_hash_join in per_partition_build_state
/// (src/include/op/sirius_physical_hash_join.hpp:409-421). It keeps a copy of the projected build
/// columns (rhs_output_columns) so a probe's gather never touches the build batch at random.
class sj_hash_table {
 public:
  sj_hash_table(cudf::table_view const& build_keys, cudf::table_view const& build_payload,
                cudf::null_equality nulls, bool unique_build_keys, rmm::cuda_stream_view stream,
                rmm::device_async_resource_ref mr);
  ~sj_hash_table();
  // not copyable or movable: the built table refers to this object's allocator context
  sj_hash_table(sj_hash_table const&)            = delete;
  sj_hash_table& operator=(sj_hash_table const&) = delete;
  sj_hash_table(sj_hash_table&&)                 = delete;
  sj_hash_table& operator=(sj_hash_table&&)      = delete;

  /// INNER probe + gather_join_output in one call: returns the output table
  /// [probe_payload columns..., build payload columns...] (src/op/sirius_physical_hash_join.cpp:1350-1355).
  std::unique_ptr<cudf::table> inner_join(cudf::table_view const& probe_keys, cudf::table_view const& probe_payload,
                                          rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr) const;

  /// The other BUILD_PROBE join types on this table (:1640-1700) with their gather:
  /// SJ_JOIN_LEFT -> [probe payload..., build payload (NULL where unmatched)...] (hash_join::left_join,
  /// distinct_hash_join::left_join + gather_distinct_left_join_output); SJ_JOIN_SEMI / SJ_JOIN_ANTI ->
  /// [probe payload...] (filtered_join::semi_join / anti_join + gather_join_output).
  std::unique_ptr<cudf::table> join(sj_join_kind kind, cudf::table_view const& probe_keys,
                                    cudf::table_view const& probe_payload, rmm::cuda_stream_view stream,
                                    rmm::device_async_resource_ref mr) const;

  /// FULL (hash_join::full_join + gather): the build columns come from the slot's retained build batch
  /// (right_full.select(rhs_output_columns)), since NULL-key build rows are not in the table.
  std::unique_ptr<cudf::table> full_join(cudf::table_view const& probe_keys, cudf::table_view const& probe_payload,
                                         cudf::table_view const& build_payload, rmm::cuda_stream_view stream,
                                         rmm::device_async_resource_ref mr) const;

  /// MARK (resolve_mark_join_result, :1461-1525): the probe columns, copied, plus a BOOL8 mark with
  /// SQL three-valued NULLs. The table must have been built with NULLs unequal.
  std::unique_ptr<cudf::table> mark_join(cudf::table_view const& probe_keys, cudf::table_view const& probe_payload,
                                         rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr) const;

 private:
  std::unique_ptr<cudf::table> run(sj_join_kind kind, cudf::table_view const& probe_keys,
                                   cudf::table_view const& probe_payload, cudf::table_view const* build_cols,
                                   rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr) const;

  rmm_alloc_ctx alloc_ctx_;  // the build's allocator context; the table frees through it
  sj_table* table_ = nullptr;
  std::vector<cudf::data_type> build_types_;
  std::vector<bool> build_nullable_;
  rmm::cuda_stream_view stream_;
};

/// The RIGHT family of STANDARD mode (src/op/sirius_physical_hash_join.cpp:1879-1895), run the way
/// the reference runs it: with the sides swapped. The table is built on the LEFT keys (the left
/// output columns attached for RIGHT) and probed with the RIGHT keys:
///   RIGHT      = cudf::left_join(right_keys, left_keys)       -> [left columns (NULL where
///                unmatched)..., right columns...]
///   RIGHT_SEMI = filtered_join(left_keys).semi_join(right)    -> [right columns...]
///   RIGHT_ANTI = filtered_join(left_keys).anti_join(right)    -> [right columns...]
/// The column order is gather_join_output's (:1299-1359): left columns, then right columns, with
/// the left side not collected for RIGHT_SEMI / RIGHT_ANTI.
enum class right_kind { RIGHT, RIGHT_SEMI, RIGHT_ANTI };
std::unique_ptr<cudf::table> right_join(right_kind kind, cudf::table_view const& left_keys,
                                        cudf::table_view const& left_cols, cudf::table_view const& right_keys,
                                        cudf::table_view const& right_cols, cudf::null_equality nulls,
                                        rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr);

}  // namespace sirius::op::sj_adapter
