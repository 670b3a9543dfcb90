// The tuning cache file: a small JSON object written and read here, so that
// the library needs no JSON dependency.
//
// {"device": "NVIDIA B200", "sm_count": 148,
//  "ops": {"scan": {"ctas_per_sm": 4, "min_rows_per_cta": 0}, "group": {...},
//          "group_i64": {...}, "probe": {...}, "topk": {...}},
//  "gb_batch": {"load_factor": 0.7, "ctas_per_sm": 3, "tile_rows": 4096}}
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <sstream>

#include "tuning.h"

namespace fdb {

static const char* const kKindNames[FDB_TUNE_KINDS] = {"scan", "group", "group_i64", "probe", "topk"};

const char* tune_kind_name(int kind) { return kind >= 0 && kind < FDB_TUNE_KINDS ? kKindNames[kind] : "?"; }

static std::string quote(const std::string& s) {
  std::string o = "\"";
  for (char ch : s) {
    const unsigned char u = (unsigned char)ch;
    if (ch == '"' || ch == '\\') {
      o += '\\';
      o += ch;
    } else if (u < 0x20) {
      char b[8];
      std::snprintf(b, sizeof(b), "\\u%04x", u);
      o += b;
    } else {
      o += ch;
    }
  }
  return o + "\"";
}

std::string tuning_to_json(const TuningSet& t, const std::string& device, int sm_count) {
  std::ostringstream o;
  o << "{\"device\": " << quote(device) << ", \"sm_count\": " << sm_count << ",\n \"ops\": {";
  for (int k = 0; k < FDB_TUNE_KINDS; ++k) {
    o << (k ? ", " : "") << "\"" << kKindNames[k] << "\": {\"ctas_per_sm\": " << t.op[k].ctas_per_sm
      << ", \"min_rows_per_cta\": " << t.op[k].min_rows_per_cta << "}";
  }
  char lf[32];
  std::snprintf(lf, sizeof(lf), "%.17g", t.batch.load_factor);
  o << "},\n \"gb_batch\": {\"load_factor\": " << lf << ", \"ctas_per_sm\": " << t.batch.ctas_per_sm
    << ", \"tile_rows\": " << t.batch.tile_rows << "}}\n";
  return o.str();
}

namespace {

// A JSON value: an object, a string or a number (all this format holds).
struct JVal {
  enum Kind { kNone, kObj, kStr, kNum } kind = kNone;
  std::map<std::string, JVal> obj;
  std::string str;
  double num = 0.0;
  std::string num_text;
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  explicit JParser(const std::string& t) : s(t) {}

  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  bool eat(char ch) {
    ws();
    if (i < s.size() && s[i] == ch) {
      ++i;
      return true;
    }
    return false;
  }
  bool string(std::string* out) {
    if (!eat('"')) return false;
    out->clear();
    while (i < s.size() && s[i] != '"') {
      char ch = s[i++];
      if (ch == '\\') {
        if (i >= s.size()) return false;
        const char e = s[i++];
        if (e == 'u') {
          if (i + 4 > s.size()) return false;
          const long code = std::strtol(s.substr(i, 4).c_str(), nullptr, 16);
          i += 4;
          if (code >= 0x80) return false;  // this format writes ASCII only
          ch = (char)code;
        } else if (e == 'n') {
          ch = '\n';
        } else if (e == 't') {
          ch = '\t';
        } else {
          ch = e;  // \" \\ \/
        }
      }
      *out += ch;
    }
    return eat('"');
  }
  bool value(JVal* v, int depth) {
    if (depth > 8) return false;
    ws();
    if (i >= s.size()) return false;
    if (s[i] == '{') {
      ++i;
      v->kind = JVal::kObj;
      if (eat('}')) return true;
      do {
        std::string key;
        if (!string(&key) || !eat(':')) return false;
        JVal child;
        if (!value(&child, depth + 1)) return false;
        v->obj[key] = std::move(child);
      } while (eat(','));
      return eat('}');
    }
    if (s[i] == '"') {
      v->kind = JVal::kStr;
      return string(&v->str);
    }
    const size_t start = i;
    while (i < s.size() && (std::isdigit((unsigned char)s[i]) || s[i] == '-' || s[i] == '+' || s[i] == '.' ||
                            s[i] == 'e' || s[i] == 'E'))
      ++i;
    if (i == start) return false;
    v->kind = JVal::kNum;
    v->num_text = s.substr(start, i - start);
    char* end = nullptr;
    v->num = std::strtod(v->num_text.c_str(), &end);
    return end && *end == '\0';
  }
};

const JVal* field(const JVal& o, const char* key, JVal::Kind kind) {
  auto it = o.obj.find(key);
  if (it == o.obj.end() || it->second.kind != kind) return nullptr;
  return &it->second;
}

bool as_int(const JVal* v, int64_t lo, int64_t hi, int64_t* out) {
  if (!v) return false;
  if (v->num_text.find_first_of(".eE") != std::string::npos) return false;
  char* end = nullptr;
  const long long x = std::strtoll(v->num_text.c_str(), &end, 10);
  if (!end || *end != '\0' || x < lo || x > hi) return false;
  *out = x;
  return true;
}

}  // namespace

std::string tuning_from_json(const std::string& text, TuningSet* out, std::string* device, int* sm_count) {
  JParser p(text);
  JVal root;
  if (!p.value(&root, 0) || root.kind != JVal::kObj) return "not a JSON object";
  p.ws();
  if (p.i != text.size()) return "trailing characters after the JSON object";
  const JVal* dev = field(root, "device", JVal::kStr);
  int64_t sms = 0;
  if (!dev) return "missing \"device\"";
  if (!as_int(field(root, "sm_count", JVal::kNum), 1, 1 << 20, &sms)) return "missing or bad \"sm_count\"";
  const JVal* ops = field(root, "ops", JVal::kObj);
  if (!ops) return "missing \"ops\"";
  TuningSet t;
  for (int k = 0; k < FDB_TUNE_KINDS; ++k) {
    const JVal* o = field(*ops, kKindNames[k], JVal::kObj);
    if (!o) continue;  // a kind the file does not tune keeps its defaults
    int64_t cps = 0, mr = 0;
    if (!as_int(field(*o, "ctas_per_sm", JVal::kNum), 0, 64, &cps))
      return std::string("bad \"ctas_per_sm\" for ") + kKindNames[k];
    if (!as_int(field(*o, "min_rows_per_cta", JVal::kNum), 0, (int64_t)1 << 40, &mr))
      return std::string("bad \"min_rows_per_cta\" for ") + kKindNames[k];
    t.op[k].ctas_per_sm = (int)cps;
    t.op[k].min_rows_per_cta = (uint64_t)mr;
  }
  if (const JVal* b = field(root, "gb_batch", JVal::kObj)) {
    const JVal* lf = field(*b, "load_factor", JVal::kNum);
    int64_t cps = 0, tr = 0;
    if (!lf || !(lf->num >= 0.0 && lf->num < 1.0)) return "bad \"gb_batch\".\"load_factor\"";
    if (!as_int(field(*b, "ctas_per_sm", JVal::kNum), 0, 64, &cps)) return "bad \"gb_batch\".\"ctas_per_sm\"";
    if (!as_int(field(*b, "tile_rows", JVal::kNum), 0, 1 << 24, &tr)) return "bad \"gb_batch\".\"tile_rows\"";
    t.batch.load_factor = lf->num;
    t.batch.ctas_per_sm = (int32_t)cps;
    t.batch.tile_rows = (int32_t)tr;
  }
  *out = t;
  *device = dev->str;
  *sm_count = (int)sms;
  return "";
}

}  // namespace fdb
