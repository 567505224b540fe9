// Stand-in: the cuDF vocabulary types the adapter uses.
#pragma once
#include <cstdint>
namespace cudf {
using size_type    = int32_t;
using bitmask_type = uint32_t;
enum class type_id : int32_t {
  EMPTY, INT8, INT16, INT32, INT64, UINT8, UINT16, UINT32, UINT64, FLOAT32, FLOAT64, BOOL8,
  TIMESTAMP_DAYS, TIMESTAMP_SECONDS, TIMESTAMP_MILLISECONDS, TIMESTAMP_MICROSECONDS,
  TIMESTAMP_NANOSECONDS, DURATION_DAYS, DURATION_SECONDS, DURATION_MILLISECONDS,
  DURATION_MICROSECONDS, DURATION_NANOSECONDS, DICTIONARY32, STRING, LIST, DECIMAL32, DECIMAL64,
  DECIMAL128, STRUCT, NUM_TYPE_IDS
};
class data_type {
 public:
  explicit constexpr data_type(type_id id) : id_(id) {}
  [[nodiscard]] constexpr type_id id() const noexcept { return id_; }
 private:
  type_id id_;
};
enum class null_equality : bool { EQUAL, UNEQUAL };
}  // namespace cudf
