// grmhd_pack.cpp - C++23 host side of the packed-GRMHD ingestion in
// include/bh_rt.h: the metadata reader (a small JSON parser for the
// nubhlight_pack schema), the blob reader with its FNV-1a 64 checksum, and the
// launch of the device resampling.
#include <cuda_runtime_api.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <variant>
#include <vector>

#include "../../../include/bh_rt.h"
#include "../device/launch.h"

namespace {

int fail(const std::string &msg) { return bhh_fail(("packed GRMHD: " + msg).c_str()); }

// ---- JSON (objects, arrays, strings, numbers, true / false / null) ---------

struct Json;
using JsonObject = std::map<std::string, Json>;
using JsonArray = std::vector<Json>;
struct Json {
  std::variant<std::nullptr_t, bool, double, std::string, JsonArray, JsonObject> v;
  bool is_num() const { return std::holds_alternative<double>(v); }
  bool is_str() const { return std::holds_alternative<std::string>(v); }
  bool is_arr() const { return std::holds_alternative<JsonArray>(v); }
  bool is_obj() const { return std::holds_alternative<JsonObject>(v); }
  double num() const { return std::get<double>(v); }
  const std::string &str() const { return std::get<std::string>(v); }
  const JsonArray &arr() const { return std::get<JsonArray>(v); }
  const JsonObject &obj() const { return std::get<JsonObject>(v); }
};

class Parser {
 public:
  explicit Parser(const std::string &t) : s_(t) {}
  bool parse(Json &out) {
    if (!value(out, 0)) return false;
    ws();
    return i_ == s_.size();
  }

 private:
  const std::string &s_;
  size_t i_ = 0;
  void ws() {
    while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_;
  }
  bool lit(const char *w) {
    const size_t n = std::strlen(w);
    if (s_.compare(i_, n, w) != 0) return false;
    i_ += n;
    return true;
  }
  bool string(std::string &out) {
    if (i_ >= s_.size() || s_[i_] != '"') return false;
    ++i_;
    out.clear();
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\') {
        if (i_ >= s_.size()) return false;
        const char e = s_[i_++];
        switch (e) {
          case 'n': c = '\n'; break;
          case 't': c = '\t'; break;
          case 'r': c = '\r'; break;
          case 'b': c = '\b'; break;
          case 'f': c = '\f'; break;
          case 'u':  // keep ASCII, replace anything wider
            if (i_ + 4 > s_.size()) return false;
            c = static_cast<char>(std::stoi(s_.substr(i_, 4), nullptr, 16) & 0x7f);
            i_ += 4;
            break;
          default: c = e;
        }
      }
      out.push_back(c);
    }
    if (i_ >= s_.size()) return false;
    ++i_;
    return true;
  }
  bool value(Json &out, int depth) {
    if (depth > 32) return false;
    ws();
    if (i_ >= s_.size()) return false;
    const char c = s_[i_];
    if (c == '{') {
      ++i_;
      JsonObject o;
      ws();
      if (i_ < s_.size() && s_[i_] == '}') {
        ++i_;
        out.v = std::move(o);
        return true;
      }
      for (;;) {
        ws();
        std::string key;
        if (!string(key)) return false;
        ws();
        if (i_ >= s_.size() || s_[i_++] != ':') return false;
        Json val;
        if (!value(val, depth + 1)) return false;
        o[key] = std::move(val);
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == '}') {
          ++i_;
          break;
        }
        return false;
      }
      out.v = std::move(o);
      return true;
    }
    if (c == '[') {
      ++i_;
      JsonArray a;
      ws();
      if (i_ < s_.size() && s_[i_] == ']') {
        ++i_;
        out.v = std::move(a);
        return true;
      }
      for (;;) {
        Json val;
        if (!value(val, depth + 1)) return false;
        a.push_back(std::move(val));
        ws();
        if (i_ < s_.size() && s_[i_] == ',') {
          ++i_;
          continue;
        }
        if (i_ < s_.size() && s_[i_] == ']') {
          ++i_;
          break;
        }
        return false;
      }
      out.v = std::move(a);
      return true;
    }
    if (c == '"') {
      std::string str;
      if (!string(str)) return false;
      out.v = std::move(str);
      return true;
    }
    if (lit("true")) {
      out.v = true;
      return true;
    }
    if (lit("false")) {
      out.v = false;
      return true;
    }
    if (lit("null")) {
      out.v = nullptr;
      return true;
    }
    const char *begin = s_.c_str() + i_;
    char *end = nullptr;
    const double d = std::strtod(begin, &end);
    if (end == begin) return false;
    i_ += static_cast<size_t>(end - begin);
    out.v = d;
    return true;
  }
};

const Json *field(const JsonObject &o, const char *k) {
  const auto it = o.find(k);
  return it == o.end() ? nullptr : &it->second;
}

std::string upper(std::string s) {
  for (char &c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return s;
}

// FNV-1a 64 over the blob's bytes, as 16 lower-case hex digits (the
// checksum nubhlight_pack writes).
std::string fnv1a64(const std::vector<float> &data) {
  uint64_t h = 14695981039346656037ull;
  const auto *b = reinterpret_cast<const unsigned char *>(data.data());
  for (size_t i = 0; i < data.size() * sizeof(float); ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  char buf[17];
  std::snprintf(buf, sizeof(buf), "%016llx", static_cast<unsigned long long>(h));
  return buf;
}

}  // namespace

extern "C" {

int bh_grmhd_packed_read(const char *json_path, BH_PackedGrmhdInfo *info, float *host_samples,
                         int64_t capacity_floats) {
  if (!json_path || !info) return fail("NULL argument");
  namespace fs = std::filesystem;
  const fs::path meta(json_path);
  std::ifstream f(meta);
  if (!f) return fail(std::string("cannot open metadata ") + json_path);
  const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  Json root;
  if (!Parser(text).parse(root) || !root.is_obj()) return fail("metadata is not a JSON object");
  const JsonObject &o = root.obj();
  const Json *fmt = field(o, "format");
  if (fmt && (!fmt->is_str() || upper(fmt->str()) != "RGBA32F"))
    return fail("format must be RGBA32F");
  const Json *bin = field(o, "bin");
  if (!bin) bin = field(o, "binary_file");
  if (!bin || !bin->is_str() || bin->str().empty()) return fail("missing 'bin' (or 'binary_file')");
  const Json *dims = field(o, "grid_dims");
  if (!dims || !dims->is_arr() || dims->arr().size() != 3) return fail("'grid_dims' must be [n_r, n_theta, n_phi]");
  int64_t d[3];
  for (int k = 0; k < 3; ++k) {
    const Json &v = dims->arr()[k];
    if (!v.is_num() || !(v.num() >= 1.0) || v.num() != std::floor(v.num()) || v.num() > 65536.0)
      return fail("'grid_dims' entries must be positive integers");
    d[k] = static_cast<int64_t>(v.num());
  }
  BH_PackedGrmhdInfo out{};
  out.n_r = static_cast<int32_t>(d[0]);
  out.n_theta = static_cast<int32_t>(d[1]);
  out.n_phi = static_cast<int32_t>(d[2]);
  out.r_min = 1.0f;
  out.r_max = 50.0f;
  if (const Json *v = field(o, "r_min"); v && v->is_num()) out.r_min = static_cast<float>(v->num());
  if (const Json *v = field(o, "r_max"); v && v->is_num()) out.r_max = static_cast<float>(v->num());
  if (!(out.r_max > out.r_min)) return fail("r_max must exceed r_min");
  const Json *ch = field(o, "channels");
  if (ch) {
    if (!ch->is_arr() || ch->arr().size() != 4) return fail("expected 4 channels");
    for (int k = 0; k < 4; ++k) {
      const Json &c = ch->arr()[k];
      std::string name = "unknown";
      if (c.is_str())
        name = c.str();
      else if (c.is_obj())
        if (const Json *nm = field(c.obj(), "name"); nm && nm->is_str()) name = nm->str();
      std::snprintf(out.channels[k], sizeof(out.channels[k]), "%s", name.c_str());
    }
  }
  for (const char *key : {"min", "max"}) {
    const Json *arr = field(o, key);
    if (!arr || !arr->is_arr()) continue;
    float *dst = key[1] == 'i' ? out.min_value : out.max_value;
    for (size_t k = 0; k < 4 && k < arr->arr().size(); ++k)
      if (arr->arr()[k].is_num()) dst[k] = static_cast<float>(arr->arr()[k].num());
  }
  const int64_t count = d[0] * d[1] * d[2] * 4;
  const fs::path blob = meta.parent_path() / bin->str();
  std::error_code ec;
  const auto bytes = fs::file_size(blob, ec);
  if (ec) return fail("cannot read blob " + blob.string());
  if (bytes != static_cast<uintmax_t>(count) * sizeof(float))
    return fail("blob holds " + std::to_string(bytes / sizeof(float)) + " floats, grid_dims need " +
                std::to_string(count));
  const Json *sum = field(o, "checksum_fnv1a64");
  if (host_samples || sum) {
    std::vector<float> data(static_cast<size_t>(count));
    std::ifstream b(blob, std::ios::binary);
    if (!b.read(reinterpret_cast<char *>(data.data()), static_cast<std::streamsize>(bytes)))
      return fail("short read of " + blob.string());
    if (sum) {
      if (!sum->is_str()) return fail("'checksum_fnv1a64' must be a string");
      std::string want = sum->str();
      for (char &c : want) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
      const std::string got = fnv1a64(data);
      if (got != want) return fail("checksum mismatch: metadata " + want + ", blob " + got);
    }
    if (host_samples) {
      if (capacity_floats < count) return fail("host buffer holds " + std::to_string(capacity_floats) +
                                               " floats, the grid needs " + std::to_string(count));
      std::memcpy(host_samples, data.data(), static_cast<size_t>(bytes));
    }
  }
  *info = out;
  return 0;
}

void bh_packed_conversion_defaults(BH_PackedConversion *conv) {
  if (!conv) return;
  conv->n_scale = 1e5;
  conv->theta_scale = 10.0;
  conv->b_scale = 30.0;
}

int bh_grmhd_from_packed(const BH_GrmhdGrid *grid, const BH_PackedGrmhdInfo *info, const void *frame_left,
                         const void *frame_right, double alpha, const BH_PackedConversion *conv, void *stream) {
  if (!grid || !grid->cells || !info || !frame_left) return fail("NULL argument");
  if (grid->n_r < 2 || grid->n_theta < 2 || grid->n_phi < 1 || !(grid->r_max > grid->r_min) || !(grid->r_min > 0.0))
    return fail("bad target grid");
  if (info->n_r < 1 || info->n_theta < 1 || info->n_phi < 1 || !(info->r_max > info->r_min))
    return fail("bad packed dimensions");
  if (frame_right && !(alpha >= 0.0 && alpha <= 1.0)) return fail("alpha must lie in [0, 1]");
  BH_PackedConversion c;
  bh_packed_conversion_defaults(&c);
  if (conv) c = *conv;
  if (bhk_grmhd_from_packed(static_cast<float *>(const_cast<void *>(grid->cells)), grid->n_r, grid->n_theta,
                            grid->n_phi, grid->r_min, grid->r_max, static_cast<const float *>(frame_left),
                            static_cast<const float *>(frame_right), frame_right ? alpha : 0.0, info->n_r,
                            info->n_theta, info->n_phi, info->r_min, info->r_max, c.n_scale, c.theta_scale,
                            c.b_scale, stream) != 0)
    return fail(std::string("resampling launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  return 0;
}

}  // extern "C"
