// json.h -- strict JSON for the request / response / artifact boundary of the femm_gpu CLI.
//
// Accepts what the reference's StrictJsonParser accepts (gpu_solver/src/io/
// strict_json.cpp:15-283): RFC 8259 grammar with ASCII whitespace, the escapes
// \" \\ \/ \b \f \n \r \t (no \u), finite numbers only (kept with their source text),
// duplicate object keys rejected, no trailing data.  Canonical serialisation (compact,
// object keys in byte order, numbers as written) and SHA-256 bind artifacts by identity
// (CanonicalJsonSha256, :466-527) and by file bytes (Sha256Hex).
#pragma once

#include <cstdint>
#include <initializer_list>
#include <map>
#include <string>
#include <vector>

namespace fgio
{

struct Json {
  enum class Kind { Null, Bool, Number, String, Array, Object };
  Kind kind = Kind::Null;
  bool boolean = false;
  double number = 0.0;
  std::string text; // number source text, or string value
  std::vector<Json> items;
  std::map<std::string, Json> members;

  bool is(Kind k) const { return kind == k; }
  // Member of an object with the given kind, or null (with *error set).
  const Json *get(const char *name, Kind k, std::string *error) const;
};

bool ParseJson(const std::string &text, Json *out, std::string *error);
// True when `value` is an object with exactly these member names.
bool HasExactly(const Json &value, std::initializer_list<const char *> names, std::string *error);
// An integral number within int32.
bool AsInt32(const Json &value, int32_t *out);
// 64 lower-case hexadecimal digits (or any-case when lower_only is false).
bool IsSha256Hex(const std::string &s, bool lower_only = true);
std::string Canonical(const Json &value);
std::string Sha256Hex(const std::string &bytes);
// JSON string escaping for responses.
std::string Escape(const std::string &s);

} // namespace fgio
