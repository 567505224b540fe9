// Sirius-side glue for the sm_100a equi-join (see sirius_hash_join_sj.hpp).
//
// Call sites it replaces in src/op/sirius_physical_hash_join.cpp:
//   build   :1614-1615 / :1852 cudf::distinct_hash_join(...)  -> sj_hash_table(..., unique=true)
//           :1620          cudf::hash_join(...)              -> sj_hash_table(..., unique=false)
//   probe   :1671 / :1688 / :1872 inner_join(...)            -> sj_hash_table::inner_join(...)
//           left_join / semi_join / anti_join (:1640-1700)    -> sj_hash_table::join(kind, ...)
//           full_join                                         -> sj_hash_table::full_join(...)
//           semi_join + resolve_mark_join_result (:1461-1525) -> sj_hash_table::mark_join(...)
//   gather  :1945-1954 gather_join_output(...)               -> (fused into the calls above)
//   STANDARD RIGHT / RIGHT_SEMI / RIGHT_ANTI (:1879-1895)     -> right_join(...): sides swapped
#include "sirius_hash_join_sj.hpp"

#include <cuda_runtime_api.h>

#include <cstdint>
#include <string>
#include <utility>

#include "cudf/null_mask.hpp"
#include "rmm/device_buffer.hpp"

namespace sirius::op::sj_adapter {

namespace {

// sj_alloc over an RMM resource (ctx: an rmm_alloc_ctx): the join's device memory is the task's
// reservation.
void* rmm_alloc(void* ctx, size_t bytes, sj_stream_t s) {
  auto* c = static_cast<rmm_alloc_ctx*>(ctx);
  try {
    return c->mr.allocate_async(bytes, 256, rmm::cuda_stream_view(reinterpret_cast<cudaStream_t>(s)));
  } catch (...) {
    return nullptr;  // -> SJ_ERR_OOM -> rmm::out_of_memory in check()
  }
}

void rmm_free(void* ctx, void* p, size_t bytes, sj_stream_t s) {
  auto* c = static_cast<rmm_alloc_ctx*>(ctx);
  c->mr.deallocate_async(p, bytes, 256, rmm::cuda_stream_view(reinterpret_cast<cudaStream_t>(s)));
}

int width_of(sj_type t) {
  switch (t) {
    case SJ_INT8:
    case SJ_BOOL8: return 1;
    case SJ_INT16: return 2;
    case SJ_INT32:
    case SJ_FLOAT32:
    case SJ_UINT32: return 4;
    default: return 8;
  }
}

sj_stream_t raw(rmm::cuda_stream_view s) { return reinterpret_cast<sj_stream_t>(s.value()); }

}  // namespace

sj_type to_sj_type(cudf::data_type t) {
  using cudf::type_id;
  switch (t.id()) {
    case type_id::INT8: return SJ_INT8;
    case type_id::UINT8: return SJ_INT8;
    case type_id::BOOL8: return SJ_BOOL8;
    case type_id::INT16:
    case type_id::UINT16: return SJ_INT16;
    case type_id::INT32:
    case type_id::TIMESTAMP_DAYS:
    case type_id::DURATION_DAYS:
    case type_id::DECIMAL32: return SJ_INT32;
    case type_id::UINT32: return SJ_UINT32;
    case type_id::INT64:
    case type_id::TIMESTAMP_SECONDS:
    case type_id::TIMESTAMP_MILLISECONDS:
    case type_id::TIMESTAMP_MICROSECONDS:
    case type_id::TIMESTAMP_NANOSECONDS:
    case type_id::DURATION_SECONDS:
    case type_id::DURATION_MILLISECONDS:
    case type_id::DURATION_MICROSECONDS:
    case type_id::DURATION_NANOSECONDS:
    case type_id::DECIMAL64: return SJ_INT64;
    case type_id::UINT64: return SJ_UINT64;
    case type_id::FLOAT32: return SJ_FLOAT32;
    case type_id::FLOAT64: return SJ_FLOAT64;
    default: throw std::runtime_error("sj adapter: column type is not fixed-width");
  }
}

sj_column to_sj(cudf::column_view const& c) {
  sj_column s{};
  const sj_type t = to_sj_type(c.type());
  s.data            = static_cast<char const*>(c.head<void>()) + (int64_t)c.offset() * width_of(t);
  s.validity        = c.nullable() ? c.null_mask() : nullptr;
  s.validity_offset = c.offset();
  s.num_rows        = c.size();
  s.type            = t;
  return s;
}

// The equi-key columns of a condition (1..4 INT32/INT64 columns; several form a composite key).
std::vector<sj_column> key_columns(cudf::table_view const& keys) {
  if (keys.num_columns() < 1 || keys.num_columns() > 4) throw std::runtime_error("sj adapter: 1 to 4 equi-key columns");
  std::vector<sj_column> out;
  for (cudf::size_type c = 0; c < keys.num_columns(); ++c) out.push_back(to_sj(keys.column(c)));
  return out;
}

void check(sj_status st, char const* where) {
  if (st == SJ_OK) return;
  const std::string msg = std::string(where) + ": " + sj_status_string(st) + ": " + sj_last_error();
  if (st == SJ_ERR_OOM) throw rmm::out_of_memory(msg.c_str());
  throw std::runtime_error(msg);
}

sj_hash_table::sj_hash_table(cudf::table_view const& build_keys, cudf::table_view const& build_payload,
                             cudf::null_equality nulls, bool unique_build_keys, rmm::cuda_stream_view stream,
                             rmm::device_async_resource_ref mr)
  : alloc_ctx_{mr}, stream_(stream)
{
  const std::vector<sj_column> keys = key_columns(build_keys);
  std::vector<sj_column> pay;
  for (cudf::size_type c = 0; c < build_payload.num_columns(); ++c) {
    pay.push_back(to_sj(build_payload.column(c)));
    build_types_.push_back(build_payload.column(c).type());
    build_nullable_.push_back(build_payload.column(c).nullable());
  }
  sj_join_params p;
  sj_default_params(&p);
  p.layout        = unique_build_keys ? SJ_LAYOUT_DISTINCT : SJ_LAYOUT_AUTO;
  p.null_equality = nulls == cudf::null_equality::EQUAL ? SJ_NULLS_EQUAL : SJ_NULLS_UNEQUAL;
  // the table keeps this sj_alloc and frees through its context in sj_table_destroy: the context is
  // the member alloc_ctx_, which lives as long as the table
  const sj_alloc a{&alloc_ctx_, rmm_alloc, rmm_free};
  // sj_build_ex synchronizes the stream, as the operator does after building (:1622)
  check(sj_build_ex(keys.data(), (int32_t)keys.size(), pay.data(), (int32_t)pay.size(), &p, &a, raw(stream), &table_),
        "sj_build_ex");
}

sj_hash_table::~sj_hash_table() { sj_table_destroy(table_, raw(stream_)); }

std::unique_ptr<cudf::table> sj_hash_table::inner_join(cudf::table_view const& probe_keys,
                                                       cudf::table_view const& probe_payload,
                                                       rmm::cuda_stream_view stream,
                                                       rmm::device_async_resource_ref mr) const
{
  return run(SJ_JOIN_INNER, probe_keys, probe_payload, nullptr, stream, mr);
}

std::unique_ptr<cudf::table> sj_hash_table::join(sj_join_kind kind, cudf::table_view const& probe_keys,
                                                 cudf::table_view const& probe_payload,
                                                 rmm::cuda_stream_view stream,
                                                 rmm::device_async_resource_ref mr) const
{
  if (kind == SJ_JOIN_MARK) return mark_join(probe_keys, probe_payload, stream, mr);
  if (kind == SJ_JOIN_FULL) throw std::runtime_error("sj adapter: FULL needs the build columns (full_join)");
  return run(kind, probe_keys, probe_payload, nullptr, stream, mr);
}

std::unique_ptr<cudf::table> sj_hash_table::full_join(cudf::table_view const& probe_keys,
                                                      cudf::table_view const& probe_payload,
                                                      cudf::table_view const& build_payload,
                                                      rmm::cuda_stream_view stream,
                                                      rmm::device_async_resource_ref mr) const
{
  return run(SJ_JOIN_FULL, probe_keys, probe_payload, &build_payload, stream, mr);
}

std::unique_ptr<cudf::table> sj_hash_table::run(sj_join_kind kind, cudf::table_view const& probe_keys,
                                                cudf::table_view const& probe_payload,
                                                cudf::table_view const* build_cols, rmm::cuda_stream_view stream,
                                                rmm::device_async_resource_ref mr) const
{
  const std::vector<sj_column> keys = key_columns(probe_keys);
  const sj_column& key = keys[0];
  rmm_alloc_ctx ctx{mr};
  const sj_alloc a{&ctx, rmm_alloc, rmm_free};
  const bool outer_build = kind == SJ_JOIN_LEFT || kind == SJ_JOIN_FULL;  // build side NULL-padded
  const bool outer_probe = kind == SJ_JOIN_FULL;                          // probe side NULL-padded
  const bool with_build  = kind == SJ_JOIN_INNER || outer_build;

  // output size: INNER matches (a DISTINCT table never returns more than it is probed with), plus
  // every probe row for LEFT/SEMI/ANTI, plus every build row for FULL
  sj_table_info info{};
  check(sj_table_get_info(table_, &info), "sj_table_get_info");
  rmm::device_buffer d_count(sizeof(int64_t), stream, mr);
  int64_t inner = key.num_rows;
  if (info.layout != SJ_LAYOUT_DISTINCT && kind != SJ_JOIN_SEMI && kind != SJ_JOIN_ANTI) {
    check(sj_probe_count(table_, keys.data(), (int32_t)keys.size(), &a, raw(stream), static_cast<int64_t*>(d_count.data())),
          "sj_probe_count");
    cudaMemcpyAsync(&inner, d_count.data(), sizeof(int64_t), cudaMemcpyDeviceToHost, stream.value());
    cudaStreamSynchronize(stream.value());
  }
  int64_t capacity = kind == SJ_JOIN_INNER ? inner : kind == SJ_JOIN_SEMI || kind == SJ_JOIN_ANTI ? key.num_rows
                                                                                                  : inner + key.num_rows;
  if (kind == SJ_JOIN_FULL) capacity += info.build_rows;

  // outputs: [probe payload columns..., build payload columns...] plus their null masks
  std::vector<sj_column> pin, bin;
  std::vector<rmm::device_buffer> data, masks;
  std::vector<cudf::data_type> types;
  std::vector<sj_mut_column> pout, bout;
  const size_t mask_bytes = (size_t)((capacity + 31) / 32) * sizeof(uint32_t);
  auto add_out = [&](cudf::data_type t, bool nullable, std::vector<sj_mut_column>& outs) {
    const sj_type st = to_sj_type(t);
    data.emplace_back((size_t)capacity * width_of(st), stream, mr);
    masks.emplace_back(nullable ? mask_bytes : 0, stream, mr);
    types.push_back(t);
    sj_mut_column m{};
    m.data     = data.back().data();
    m.validity = nullable ? static_cast<uint32_t*>(masks.back().data()) : nullptr;
    m.type     = st;
    outs.push_back(m);
  };
  for (cudf::size_type c = 0; c < probe_payload.num_columns(); ++c) {
    pin.push_back(to_sj(probe_payload.column(c)));
    add_out(probe_payload.column(c).type(), outer_probe || probe_payload.column(c).nullable(), pout);
  }
  if (with_build && build_cols) {
    for (cudf::size_type c = 0; c < build_cols->num_columns(); ++c) {
      bin.push_back(to_sj(build_cols->column(c)));
      add_out(build_cols->column(c).type(), true, bout);
    }
  } else if (with_build) {
    for (size_t c = 0; c < build_types_.size(); ++c) add_out(build_types_[c], outer_build || build_nullable_[c], bout);
  }

  check(sj_probe_join(table_, kind, keys.data(), (int32_t)keys.size(), pin.data(), (int32_t)pin.size(),
                      build_cols ? bin.data() : nullptr /* NULL: the attached build columns */, (int32_t)bout.size(),
                      nullptr, nullptr, pout.data(), bout.data(), capacity, nullptr, nullptr, &a, raw(stream),
                      static_cast<int64_t*>(d_count.data())),
        "sj_probe_join");
  int64_t rows = 0;
  cudaMemcpyAsync(&rows, d_count.data(), sizeof(int64_t), cudaMemcpyDeviceToHost, stream.value());
  cudaStreamSynchronize(stream.value());
  if (rows > capacity) throw std::runtime_error("sj adapter: the join produced more rows than counted");

  std::vector<std::unique_ptr<cudf::column>> cols;
  for (size_t c = 0; c < data.size(); ++c) {
    const bool nullable      = masks[c].size() > 0;
    const auto n             = static_cast<cudf::size_type>(rows);
    const cudf::size_type nc = nullable ? cudf::null_count(static_cast<cudf::bitmask_type const*>(masks[c].data()),
                                                           0, n, stream)
                                        : 0;
    cols.push_back(std::make_unique<cudf::column>(types[c], n, std::move(data[c]), std::move(masks[c]), nc));
  }
  return std::make_unique<cudf::table>(std::move(cols), stream);
}

std::unique_ptr<cudf::table> sj_hash_table::mark_join(cudf::table_view const& probe_keys,
                                                      cudf::table_view const& probe_payload,
                                                      rmm::cuda_stream_view stream,
                                                      rmm::device_async_resource_ref mr) const
{
  const std::vector<sj_column> keys = key_columns(probe_keys);
  const sj_column& key = keys[0];
  rmm_alloc_ctx ctx{mr};
  const sj_alloc a{&ctx, rmm_alloc, rmm_free};
  const auto n = static_cast<cudf::size_type>(key.num_rows);
  rmm::device_buffer d_count(sizeof(int64_t), stream, mr);
  rmm::device_buffer mark((size_t)n, stream, mr);
  rmm::device_buffer mask((size_t)((n + 31) / 32) * sizeof(uint32_t), stream, mr);
  check(sj_probe_join(table_, SJ_JOIN_MARK, keys.data(), (int32_t)keys.size(), nullptr, 0, nullptr, 0, nullptr, nullptr,
                      nullptr, nullptr, 0,
                      static_cast<uint8_t*>(mark.data()), static_cast<uint32_t*>(mask.data()), &a, raw(stream),
                      static_cast<int64_t*>(d_count.data())),
        "sj_probe_join");
  std::vector<std::unique_ptr<cudf::column>> cols;
  for (cudf::size_type c = 0; c < probe_payload.num_columns(); ++c)
    cols.push_back(std::make_unique<cudf::column>(probe_payload.column(c), stream, mr));
  const cudf::size_type nc = cudf::null_count(static_cast<cudf::bitmask_type const*>(mask.data()), 0, n, stream);
  cols.push_back(std::make_unique<cudf::column>(cudf::data_type(cudf::type_id::BOOL8), n, std::move(mark),
                                                std::move(mask), nc));
  return std::make_unique<cudf::table>(std::move(cols), stream);
}

std::unique_ptr<cudf::table> right_join(right_kind kind, cudf::table_view const& left_keys,
                                        cudf::table_view const& left_cols, cudf::table_view const& right_keys,
                                        cudf::table_view const& right_cols, cudf::null_equality nulls,
                                        rmm::cuda_stream_view stream, rmm::device_async_resource_ref mr)
{
  const bool collect_left = kind == right_kind::RIGHT;
  // build on the left side (its projected columns attached only when they are output)
  const sj_hash_table table(left_keys, collect_left ? left_cols : cudf::table_view{}, nulls,
                            /*unique_build_keys=*/false, stream, mr);
  if (!collect_left)
    return table.join(kind == right_kind::RIGHT_SEMI ? SJ_JOIN_SEMI : SJ_JOIN_ANTI, right_keys, right_cols, stream, mr);
  // LEFT join of right over left gives [right columns..., left columns (NULL-padded)...]
  auto swapped = table.join(SJ_JOIN_LEFT, right_keys, right_cols, stream, mr);
  auto cols    = swapped->release();
  std::vector<std::unique_ptr<cudf::column>> out;
  const size_t n_right = static_cast<size_t>(right_cols.num_columns());
  for (size_t c = n_right; c < cols.size(); ++c) out.push_back(std::move(cols[c]));
  for (size_t c = 0; c < n_right; ++c) out.push_back(std::move(cols[c]));
  return std::make_unique<cudf::table>(std::move(out), stream);
}

}  // namespace sirius::op::sj_adapter
