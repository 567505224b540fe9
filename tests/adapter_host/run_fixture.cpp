// Runs the Sirius adapter (adapter/sirius_hash_join_sj.cpp) end to end on the GPU over the
// reference's NULL-join fixture (test/cpp/integration/test_gpu_execution_join_nulls.cpp:37-43) and
// prints every result as one JSON line per case, for tests/test_gpu_adapter.py to compare with the
// known answers.
//
// stdin:
//   L id:k id:k ...      left rows (k = N for NULL); int32 ids and keys
//   R id:k id:k ...      right rows
//   M name keys keys     a MARK case: left keys, right keys (comma separated, N = NULL, - = none)
// Each case builds its table, probes, reads the result back and destroys the table (so every
// sj_hash_table destructor runs, freeing through the allocator context it was built with).
// Finally an allocation-refusal sweep: the Nth device allocation of a build + INNER probe is
// refused, for every N until the join succeeds; each refusal must surface as rmm::out_of_memory
// with no device allocation left alive.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include "sirius_hash_join_sj.hpp"
#include "standin_runtime.hpp"

extern "C" cudaError_t cudaMemcpy(void* dst, const void* src, size_t count, enum cudaMemcpyKind kind);
extern "C" cudaError_t cudaDeviceSynchronize(void);

namespace sa = sirius::op::sj_adapter;
using cudf::column_view;
using cudf::data_type;
using cudf::table_view;
using cudf::type_id;

namespace {

// A host column uploaded to the device; keeps its buffers alive.
struct dev_col {
  dev_col(size_t data_bytes, size_t mask_bytes, rmm::cuda_stream_view s) : data(data_bytes, s), mask(mask_bytes, s) {}
  rmm::device_buffer data, mask;
  column_view view;
};

std::unique_ptr<dev_col> upload(std::vector<std::optional<int32_t>> const& v, rmm::cuda_stream_view s) {
  const size_t n = v.size();
  std::vector<int32_t> h(n, 0);
  std::vector<uint32_t> m((n + 31) / 32 + 1, 0);
  auto c = std::make_unique<dev_col>(n * 4 + 4, m.size() * 4, s);
  int nulls = 0;
  for (size_t i = 0; i < n; ++i) {
    if (v[i]) {
      h[i] = *v[i];
      m[i / 32] |= 1u << (i % 32);
    } else {
      ++nulls;
    }
  }
  s.synchronize();
  cudaMemcpy(c->data.data(), h.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(c->mask.data(), m.data(), m.size() * 4, cudaMemcpyHostToDevice);
  c->view = column_view(data_type(type_id::INT32), static_cast<cudf::size_type>(n), c->data.data(),
                        nulls ? static_cast<cudf::bitmask_type const*>(c->mask.data()) : nullptr, nulls);
  return c;
}

// One value of a result column as JSON (null for NULL).
std::vector<std::string> download(column_view const& c) {
  const int w = standin::width_of(c.type());
  const size_t n = static_cast<size_t>(c.size());
  std::vector<unsigned char> h(n * w + 8);
  std::vector<uint32_t> m((n + 31) / 32 + 1, ~0u);
  cudaDeviceSynchronize();
  if (n) cudaMemcpy(h.data(), c.head(), n * w, cudaMemcpyDeviceToHost);
  if (n && c.nullable()) cudaMemcpy(m.data(), c.null_mask(), (n + 31) / 32 * 4, cudaMemcpyDeviceToHost);
  std::vector<std::string> out;
  for (size_t i = 0; i < n; ++i) {
    if (!((m[i / 32] >> (i % 32)) & 1u)) {
      out.emplace_back("null");
    } else if (c.type().id() == type_id::BOOL8) {
      out.emplace_back(h[i] ? "true" : "false");
    } else {
      int32_t x;
      std::memcpy(&x, &h[i * 4], 4);
      out.push_back(std::to_string(x));
    }
  }
  return out;
}

void print_rows(std::string const& name, cudf::table const& t) {
  std::vector<std::vector<std::string>> cols;
  for (cudf::size_type c = 0; c < t.num_columns(); ++c) cols.push_back(download(t.get_column(c).view()));
  std::ostringstream o;
  o << "{\"case\": \"" << name << "\", \"rows\": [";
  for (cudf::size_type r = 0; r < t.num_rows(); ++r) {
    o << (r ? ", [" : "[");
    for (size_t c = 0; c < cols.size(); ++c) o << (c ? ", " : "") << cols[c][r];
    o << "]";
  }
  o << "], \"live_allocations\": " << standin::current().live << "}";
  std::cout << o.str() << std::endl;
}

std::vector<std::optional<int32_t>> parse_keys(std::string const& s) {
  std::vector<std::optional<int32_t>> v;
  if (s == "-") return v;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ',')) {
    if (tok == "N") v.emplace_back(std::nullopt);
    else v.emplace_back(std::stoi(tok));
  }
  return v;
}

void parse_side(std::string const& line, std::vector<std::optional<int32_t>>& id, std::vector<std::optional<int32_t>>& k) {
  std::stringstream ss(line.substr(2));
  std::string tok;
  while (ss >> tok) {
    const auto c = tok.find(':');
    id.emplace_back(std::stoi(tok.substr(0, c)));
    const std::string kk = tok.substr(c + 1);
    if (kk == "N") k.emplace_back(std::nullopt);
    else k.emplace_back(std::stoi(kk));
  }
}

}  // namespace

int main() {
  const rmm::cuda_stream_view s{};
  auto mr = rmm::mr::get_current_device_resource_ref();
  std::vector<std::optional<int32_t>> lid, lk, rid, rk;
  std::vector<std::string> mark_lines;
  std::string line;
  while (std::getline(std::cin, line)) {
    if (line.rfind("L ", 0) == 0) parse_side(line, lid, lk);
    else if (line.rfind("R ", 0) == 0) parse_side(line, rid, rk);
    else if (line.rfind("M ", 0) == 0) mark_lines.push_back(line);
  }
  try {
    auto L_id = upload(lid, s), L_k = upload(lk, s), R_id = upload(rid, s), R_k = upload(rk, s);
    const table_view lkeys({L_k->view}), lcols({L_id->view}), rkeys({R_k->view}), rcols({R_id->view});
    const table_view none;
    // BUILD_PROBE on the right side, probed by the left: INNER, LEFT, SEMI, ANTI, FULL, MARK
    {
      sa::sj_hash_table t(rkeys, rcols, cudf::null_equality::UNEQUAL, false, s, mr);
      print_rows("inner", *t.inner_join(lkeys, lcols, s, mr));
      print_rows("left", *t.join(SJ_JOIN_LEFT, lkeys, lcols, s, mr));
      print_rows("full", *t.full_join(lkeys, lcols, rcols, s, mr));
    }
    {
      sa::sj_hash_table t(rkeys, none, cudf::null_equality::UNEQUAL, false, s, mr);
      print_rows("semi", *t.join(SJ_JOIN_SEMI, lkeys, lcols, s, mr));
      print_rows("anti", *t.join(SJ_JOIN_ANTI, lkeys, lcols, s, mr));
      print_rows("mark_with_null_build", *t.mark_join(lkeys, lcols, s, mr));
    }
    {
      sa::sj_hash_table t(rkeys, rcols, cudf::null_equality::EQUAL, false, s, mr);
      print_rows("inner_null_safe", *t.inner_join(lkeys, lcols, s, mr));
    }
    // STANDARD-mode RIGHT family: sides swapped (build on the left)
    print_rows("right", *sa::right_join(sa::right_kind::RIGHT, lkeys, lcols, rkeys, rcols,
                                        cudf::null_equality::UNEQUAL, s, mr));
    print_rows("right_semi", *sa::right_join(sa::right_kind::RIGHT_SEMI, lkeys, lcols, rkeys, rcols,
                                             cudf::null_equality::UNEQUAL, s, mr));
    print_rows("right_anti", *sa::right_join(sa::right_kind::RIGHT_ANTI, lkeys, lcols, rkeys, rcols,
                                             cudf::null_equality::UNEQUAL, s, mr));
    // the operator-level MARK cases
    for (auto const& ml : mark_lines) {
      std::stringstream ss(ml.substr(2));
      std::string name, lks, rks;
      ss >> name >> lks >> rks;
      auto lv = parse_keys(lks), rv = parse_keys(rks);
      std::vector<std::optional<int32_t>> ids;
      for (size_t i = 0; i < lv.size(); ++i) ids.emplace_back(static_cast<int32_t>(i));
      auto mk = upload(lv, s), mi = upload(ids, s), bk = upload(rv, s);
      sa::sj_hash_table t(table_view({bk->view}), none, cudf::null_equality::UNEQUAL, false, s, mr);
      print_rows("mark:" + name, *t.mark_join(table_view({mk->view}), table_view({mi->view}), s, mr));
    }
  } catch (std::exception const& e) {
    std::cout << "{\"case\": \"error\", \"what\": \"" << e.what() << "\"}" << std::endl;
    return 1;
  }
  // allocation refusals: the Nth allocation of (upload, build, probe, output) fails
  std::ostringstream o;
  o << "{\"case\": \"oom_sweep\", \"attempts\": [";
  auto& led = standin::current();
  bool first = true;
  for (int n = 1; n <= 64; ++n) {
    const int64_t live0 = led.live;
    led.calls = 0;
    led.fail_at = n;
    std::string outcome;
    try {
      auto L_k = upload(lk, s), L_id = upload(lid, s), R_k = upload(rk, s), R_id = upload(rid, s);
      sa::sj_hash_table t(table_view({R_k->view}), table_view({R_id->view}), cudf::null_equality::UNEQUAL, false, s, mr);
      auto out = t.inner_join(table_view({L_k->view}), table_view({L_id->view}), s, mr);
      outcome = "ok:" + std::to_string(out->num_rows());
    } catch (rmm::out_of_memory const&) {
      outcome = "oom";
    } catch (std::exception const& e) {
      outcome = std::string("other:") + e.what();
    }
    cudaDeviceSynchronize();
    o << (first ? "" : ", ") << "{\"fail_at\": " << n << ", \"outcome\": \"" << outcome
      << "\", \"leaked\": " << (led.live - live0) << "}";
    first = false;
    if (outcome.rfind("ok:", 0) == 0) break;
  }
  led.fail_at = 0;
  o << "], \"live_allocations\": " << led.live << "}";
  std::cout << o.str() << std::endl;
  return 0;
}
