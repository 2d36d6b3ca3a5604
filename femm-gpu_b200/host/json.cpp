// json.cpp -- strict JSON parser, canonical form and SHA-256 (FIPS 180-4).
#include "json.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>

namespace fgio
{
namespace
{

bool Space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }
bool Digit(char c) { return c >= '0' && c <= '9'; }

class Parser
{
public:
  explicit Parser(const std::string &s) : s_(s) {}

  bool Document(Json *out, std::string *error)
  {
    SkipSpace();
    if (!Value(out, error))
      return false;
    SkipSpace();
    if (at_ != s_.size())
      return Fail(error, "trailing JSON data");
    return true;
  }

private:
  bool Fail(std::string *error, const char *what)
  {
    *error = what;
    return false;
  }
  void SkipSpace()
  {
    while (at_ < s_.size() && Space(s_[at_]))
      ++at_;
  }
  bool Word(const char *w)
  {
    const size_t n = std::strlen(w);
    if (s_.compare(at_, n, w) != 0)
      return false;
    at_ += n;
    return true;
  }

  bool Value(Json *v, std::string *error)
  {
    if (at_ >= s_.size())
      return Fail(error, "unexpected JSON end");
    switch (s_[at_]) {
    case '{':
      return Object(v, error);
    case '[':
      return Array(v, error);
    case '"':
      v->kind = Json::Kind::String;
      return String(&v->text, error);
    default:
      break;
    }
    if (Word("true")) {
      v->kind = Json::Kind::Bool;
      v->boolean = true;
      return true;
    }
    if (Word("false")) {
      v->kind = Json::Kind::Bool;
      v->boolean = false;
      return true;
    }
    if (Word("null")) {
      v->kind = Json::Kind::Null;
      return true;
    }
    return Number(v, error);
  }

  bool String(std::string *out, std::string *error)
  {
    ++at_; // opening quote
    out->clear();
    while (at_ < s_.size()) {
      const unsigned char c = static_cast<unsigned char>(s_[at_++]);
      if (c == '"')
        return true;
      if (c < 0x20)
        return Fail(error, "control character in JSON string");
      if (c != '\\') {
        out->push_back(static_cast<char>(c));
        continue;
      }
      if (at_ >= s_.size())
        return Fail(error, "truncated JSON escape");
      static const char from[] = "\"\\/bfnrt";
      static const char to[] = "\"\\/\b\f\n\r\t";
      const char *hit = std::strchr(from, s_[at_]);
      if (!hit || *hit == '\0')
        return Fail(error, "unsupported JSON string escape");
      out->push_back(to[hit - from]);
      ++at_;
    }
    return Fail(error, "unterminated JSON string");
  }

  bool Number(Json *v, std::string *error)
  {
    const size_t begin = at_;
    if (at_ < s_.size() && s_[at_] == '-')
      ++at_;
    if (at_ >= s_.size())
      return Fail(error, "invalid JSON number");
    if (s_[at_] == '0') {
      ++at_;
    } else if (s_[at_] >= '1' && s_[at_] <= '9') {
      while (at_ < s_.size() && Digit(s_[at_]))
        ++at_;
    } else {
      return Fail(error, "invalid JSON number");
    }
    if (at_ < s_.size() && s_[at_] == '.') {
      const size_t f = ++at_;
      while (at_ < s_.size() && Digit(s_[at_]))
        ++at_;
      if (at_ == f)
        return Fail(error, "invalid JSON fraction");
    }
    if (at_ < s_.size() && (s_[at_] == 'e' || s_[at_] == 'E')) {
      ++at_;
      if (at_ < s_.size() && (s_[at_] == '+' || s_[at_] == '-'))
        ++at_;
      const size_t e = at_;
      while (at_ < s_.size() && Digit(s_[at_]))
        ++at_;
      if (at_ == e)
        return Fail(error, "invalid JSON exponent");
    }
    v->kind = Json::Kind::Number;
    v->text = s_.substr(begin, at_ - begin);
    // Conversion as std::stod does it: an out-of-range magnitude is an error.
    errno = 0;
    char *end = nullptr;
    const double d = std::strtod(v->text.c_str(), &end);
    if (end != v->text.c_str() + v->text.size() || errno == ERANGE)
      return Fail(error, "JSON number conversion failed");
    if (!std::isfinite(d))
      return Fail(error, "nonfinite JSON number");
    v->number = d;
    return true;
  }

  bool Array(Json *v, std::string *error)
  {
    ++at_;
    v->kind = Json::Kind::Array;
    v->items.clear();
    SkipSpace();
    if (at_ < s_.size() && s_[at_] == ']') {
      ++at_;
      return true;
    }
    for (;;) {
      v->items.emplace_back();
      if (!Value(&v->items.back(), error))
        return false;
      SkipSpace();
      if (at_ >= s_.size())
        return Fail(error, "unterminated JSON array");
      const char c = s_[at_++];
      if (c == ']')
        return true;
      if (c != ',')
        return Fail(error, "JSON array comma expected");
      SkipSpace();
    }
  }

  bool Object(Json *v, std::string *error)
  {
    ++at_;
    v->kind = Json::Kind::Object;
    v->members.clear();
    SkipSpace();
    if (at_ < s_.size() && s_[at_] == '}') {
      ++at_;
      return true;
    }
    for (;;) {
      std::string key;
      if (at_ >= s_.size() || s_[at_] != '"' || !String(&key, error))
        return Fail(error, "JSON object key expected");
      SkipSpace();
      if (at_ >= s_.size() || s_[at_++] != ':')
        return Fail(error, "JSON colon expected");
      SkipSpace();
      Json child;
      if (!Value(&child, error))
        return false;
      if (!v->members.emplace(std::move(key), std::move(child)).second)
        return Fail(error, "duplicate JSON object key");
      SkipSpace();
      if (at_ >= s_.size())
        return Fail(error, "unterminated JSON object");
      const char c = s_[at_++];
      if (c == '}')
        return true;
      if (c != ',')
        return Fail(error, "JSON object comma expected");
      SkipSpace();
    }
  }

  const std::string &s_;
  size_t at_ = 0;
};

void AppendCanonical(const Json &v, std::string *out)
{
  switch (v.kind) {
  case Json::Kind::Null:
    out->append("null");
    break;
  case Json::Kind::Bool:
    out->append(v.boolean ? "true" : "false");
    break;
  case Json::Kind::Number:
    out->append(v.text);
    break;
  case Json::Kind::String:
    out->push_back('"');
    out->append(Escape(v.text));
    out->push_back('"');
    break;
  case Json::Kind::Array:
    out->push_back('[');
    for (size_t i = 0; i < v.items.size(); ++i) {
      if (i)
        out->push_back(',');
      AppendCanonical(v.items[i], out);
    }
    out->push_back(']');
    break;
  case Json::Kind::Object: {
    out->push_back('{');
    bool first = true;
    for (const auto &m : v.members) { // std::map<std::string>: byte order
      if (!first)
        out->push_back(',');
      first = false;
      out->push_back('"');
      out->append(Escape(m.first));
      out->append("\":");
      AppendCanonical(m.second, out);
    }
    out->push_back('}');
    break;
  }
  }
}

// SHA-256 as specified in FIPS 180-4 (sections 4.1.2, 4.2.2, 5.3.3, 6.2).
struct Sha256State {
  uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                   0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};

  static uint32_t Rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

  void Block(const unsigned char *p)
  {
    static const uint32_t K[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
        0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
        0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
        0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
        0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
        0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    uint32_t w[64];
    for (int t = 0; t < 16; ++t)
      w[t] = uint32_t(p[4 * t]) << 24 | uint32_t(p[4 * t + 1]) << 16 | uint32_t(p[4 * t + 2]) << 8 | p[4 * t + 3];
    for (int t = 16; t < 64; ++t) {
      const uint32_t s0 = Rotr(w[t - 15], 7) ^ Rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
      const uint32_t s1 = Rotr(w[t - 2], 17) ^ Rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
      w[t] = s1 + w[t - 7] + s0 + w[t - 16];
    }
    uint32_t v[8];
    std::memcpy(v, h, sizeof(v));
    for (int t = 0; t < 64; ++t) {
      const uint32_t big1 = Rotr(v[4], 6) ^ Rotr(v[4], 11) ^ Rotr(v[4], 25);
      const uint32_t choose = (v[4] & v[5]) ^ (~v[4] & v[6]);
      const uint32_t t1 = v[7] + big1 + choose + K[t] + w[t];
      const uint32_t big0 = Rotr(v[0], 2) ^ Rotr(v[0], 13) ^ Rotr(v[0], 22);
      const uint32_t major = (v[0] & v[1]) ^ (v[0] & v[2]) ^ (v[1] & v[2]);
      for (int i = 7; i > 0; --i)
        v[i] = v[i - 1];
      v[4] += t1;
      v[0] = t1 + big0 + major;
    }
    for (int i = 0; i < 8; ++i)
      h[i] += v[i];
  }
};

} // namespace

const Json *Json::get(const char *name, Kind k, std::string *error) const
{
  if (kind != Kind::Object) {
    *error = "expected JSON object";
    return nullptr;
  }
  const auto it = members.find(name);
  if (it == members.end()) {
    *error = std::string("missing JSON field: ") + name;
    return nullptr;
  }
  if (it->second.kind != k) {
    *error = std::string("wrong JSON type: ") + name;
    return nullptr;
  }
  return &it->second;
}

bool ParseJson(const std::string &text, Json *out, std::string *error)
{
  Parser p(text);
  *out = Json{};
  return p.Document(out, error);
}

bool HasExactly(const Json &value, std::initializer_list<const char *> names, std::string *error)
{
  if (value.kind != Json::Kind::Object || value.members.size() != names.size()) {
    *error = "unexpected JSON object fields";
    return false;
  }
  for (const char *n : names)
    if (!value.members.count(n)) {
      *error = std::string("missing JSON field: ") + n;
      return false;
    }
  return true;
}

bool AsInt32(const Json &value, int32_t *out)
{
  if (value.kind != Json::Kind::Number || value.number != std::floor(value.number) ||
      value.number < double(std::numeric_limits<int32_t>::min()) ||
      value.number > double(std::numeric_limits<int32_t>::max()))
    return false;
  *out = static_cast<int32_t>(value.number);
  return true;
}

bool IsSha256Hex(const std::string &s, bool lower_only)
{
  if (s.size() != 64)
    return false;
  for (char c : s) {
    const bool ok = Digit(c) || (c >= 'a' && c <= 'f') || (!lower_only && c >= 'A' && c <= 'F');
    if (!ok)
      return false;
  }
  return true;
}

std::string Canonical(const Json &value)
{
  std::string out;
  AppendCanonical(value, &out);
  return out;
}

std::string Sha256Hex(const std::string &bytes)
{
  Sha256State st;
  const size_t n = bytes.size();
  const auto *data = reinterpret_cast<const unsigned char *>(bytes.data());
  size_t i = 0;
  for (; i + 64 <= n; i += 64)
    st.Block(data + i);
  unsigned char tail[128] = {};
  const size_t rest = n - i;
  std::memcpy(tail, data + i, rest);
  tail[rest] = 0x80;
  const size_t blocks = rest + 1 + 8 <= 64 ? 1 : 2;
  const uint64_t bits = static_cast<uint64_t>(n) * 8;
  for (int b = 0; b < 8; ++b)
    tail[blocks * 64 - 1 - b] = static_cast<unsigned char>(bits >> (8 * b));
  for (size_t b = 0; b < blocks; ++b)
    st.Block(tail + 64 * b);
  char hex[65];
  for (int w = 0; w < 8; ++w)
    std::snprintf(hex + 8 * w, 9, "%08x", st.h[w]);
  return std::string(hex, 64);
}

std::string Escape(const std::string &s)
{
  std::string out;
  for (unsigned char c : s) {
    switch (c) {
    case '"': out += "\\\""; break;
    case '\\': out += "\\\\"; break;
    case '\b': out += "\\b"; break;
    case '\f': out += "\\f"; break;
    case '\n': out += "\\n"; break;
    case '\r': out += "\\r"; break;
    case '\t': out += "\\t"; break;
    default:
      if (c < 0x20) {
        char buf[8];
        std::snprintf(buf, sizeof(buf), "\\u%04x", c);
        out += buf;
      } else {
        out.push_back(static_cast<char>(c));
      }
    }
  }
  return out;
}

} // namespace fgio
