// vfb_io.cpp -- trace JSON reader and infix printer of the C ABI.
//
// The reader accepts the reference's schema (readJsonFile ltl_nocache.cu:35-76)
// with a small recursive-descent JSON parser of its own.  Encoding follows the
// reference: trace i's length is the length of its first proposition's array
// (ltl_nocache.cu:57); proposition v's bit t is set when values[t] != 0
// (ltl_nocache.cu:58-65); positives come first.  Inputs the reference would
// read out of bounds (declared counts that disagree with the arrays, arrays
// longer than 64 steps, missing propositions) are rejected with an error.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vfb.h"

namespace {

struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  double num = 0;
  bool b = false;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const std::string& k) const {
    for (const auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct Parser {
  const char* p;
  const char* end;
  std::string err;
  int depth = 0;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
  }
  bool fail(const char* m) {
    if (err.empty()) err = m;
    return false;
  }
  bool lit(const char* s) {
    const size_t n = std::strlen(s);
    if ((size_t)(end - p) < n || std::strncmp(p, s, n) != 0) return false;
    p += n;
    return true;
  }
  bool string(std::string& out) {
    if (p >= end || *p != '"') return fail("expected string");
    ++p;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) return fail("bad escape");
        switch (*p) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (end - p < 5) return fail("bad \\u escape");
            unsigned code = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
            if (code < 0x80) {
              out += (char)code;
            } else if (code < 0x800) {
              out += (char)(0xC0 | (code >> 6));
              out += (char)(0x80 | (code & 0x3F));
            } else {
              out += (char)(0xE0 | (code >> 12));
              out += (char)(0x80 | ((code >> 6) & 0x3F));
              out += (char)(0x80 | (code & 0x3F));
            }
            p += 4;
            break;
          }
          default: out += *p;
        }
        ++p;
      } else {
        out += *p++;
      }
    }
    if (p >= end) return fail("unterminated string");
    ++p;
    return true;
  }
  bool value(JVal& v) {
    if (++depth > 64) return fail("nesting too deep");
    ws();
    if (p >= end) return fail("unexpected end");
    bool ok = true;
    if (*p == '{') {
      v.kind = JVal::OBJ;
      ++p;
      ws();
      if (p < end && *p == '}') {
        ++p;
      } else {
        while (ok) {
          ws();
          std::string k;
          if (!string(k)) { ok = false; break; }
          ws();
          if (p >= end || *p != ':') { ok = fail("expected ':'"); break; }
          ++p;
          JVal x;
          if (!value(x)) { ok = false; break; }
          v.obj.emplace_back(std::move(k), std::move(x));
          ws();
          if (p < end && *p == ',') { ++p; continue; }
          if (p < end && *p == '}') { ++p; break; }
          ok = fail("expected ',' or '}'");
        }
      }
    } else if (*p == '[') {
      v.kind = JVal::ARR;
      ++p;
      ws();
      if (p < end && *p == ']') {
        ++p;
      } else {
        while (ok) {
          JVal x;
          if (!value(x)) { ok = false; break; }
          v.arr.push_back(std::move(x));
          ws();
          if (p < end && *p == ',') { ++p; continue; }
          if (p < end && *p == ']') { ++p; break; }
          ok = fail("expected ',' or ']'");
        }
      }
    } else if (*p == '"') {
      v.kind = JVal::STR;
      ok = string(v.str);
    } else if (lit("true")) {
      v.kind = JVal::BOOL;
      v.b = true;
    } else if (lit("false")) {
      v.kind = JVal::BOOL;
    } else if (lit("null")) {
      v.kind = JVal::NUL;
    } else if (*p == '-' || std::isdigit((unsigned char)*p)) {
      char* q = nullptr;
      v.kind = JVal::NUM;
      v.num = std::strtod(p, &q);
      if (q == p) ok = fail("bad number");
      p = q;
    } else {
      ok = fail("unexpected character");
    }
    --depth;
    return ok;
  }
};

void set_err(char* err, size_t n, const std::string& m) {
  if (err && n) std::snprintf(err, n, "%s", m.c_str());
}

bool as_int(const JVal* v, long long& out) {
  if (!v || v->kind != JVal::NUM) return false;
  out = (long long)v->num;
  return (double)out == v->num;
}

struct Owned : vfb_json_problem {
  std::vector<uint64_t> words;
  std::vector<int> lengths;
  std::vector<std::string> names;
  std::vector<char*> name_ptrs;
};

}  // namespace

extern "C" {

vfb_status vfb_read_json(const char* path, vfb_json_problem** out, char* err, size_t errlen) {
  if (!path || !out) return VFB_BAD_INPUT;
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_err(err, errlen, std::string("Error: Could not open file ") + path);
    return VFB_BAD_INPUT;
  }
  std::string text;
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  std::fclose(f);
  Parser ps{text.data(), text.data() + text.size()};
  JVal root;
  if (!ps.value(root) || root.kind != JVal::OBJ) {
    set_err(err, errlen, "JSON parse error: " + (ps.err.empty() ? std::string("not an object") : ps.err));
    return VFB_BAD_INPUT;
  }
  long long nvar, ntr, npos, maxlen;
  if (!as_int(root.get("number_atomic_propositions"), nvar) || !as_int(root.get("number_traces"), ntr) ||
      !as_int(root.get("number_positive_traces"), npos) || !as_int(root.get("max_length_traces"), maxlen)) {
    set_err(err, errlen, "missing or non-integer count fields");
    return VFB_BAD_INPUT;
  }
  const JVal* aps = root.get("atomic_propositions");
  const JVal* pos = root.get("positive_traces");
  const JVal* neg = root.get("negative_traces");
  if (!aps || aps->kind != JVal::ARR || !pos || pos->kind != JVal::ARR || !neg || neg->kind != JVal::ARR) {
    set_err(err, errlen, "missing atomic_propositions / positive_traces / negative_traces");
    return VFB_BAD_INPUT;
  }
  if (nvar < 1 || (long long)aps->arr.size() < nvar) {
    set_err(err, errlen, "atomic_propositions has fewer names than number_atomic_propositions");
    return VFB_BAD_INPUT;
  }
  if ((long long)(pos->arr.size() + neg->arr.size()) != ntr || (long long)pos->arr.size() != npos) {
    set_err(err, errlen, "trace counts disagree with number_traces / number_positive_traces");
    return VFB_BAD_INPUT;
  }
  std::unique_ptr<Owned> o(new Owned());
  static_cast<vfb_json_problem&>(*o) = vfb_json_problem{};
  for (long long v = 0; v < nvar; ++v) {
    if (aps->arr[v].kind != JVal::STR) {
      set_err(err, errlen, "proposition names must be strings");
      return VFB_BAD_INPUT;
    }
    o->names.push_back(aps->arr[v].str);
  }
  o->words.assign((size_t)ntr * nvar, 0ULL);
  o->lengths.assign((size_t)ntr, 0);
  long long idx = 0;
  for (const JVal* set : {pos, neg}) {
    for (const JVal& tr : set->arr) {
      if (tr.kind != JVal::OBJ) {
        set_err(err, errlen, "a trace is not an object");
        return VFB_BAD_INPUT;
      }
      for (long long v = 0; v < nvar; ++v) {
        const JVal* vals = tr.get(o->names[v]);
        if (!vals || vals->kind != JVal::ARR) {
          set_err(err, errlen, "trace " + std::to_string(idx) + " lacks proposition " + o->names[v]);
          return VFB_BAD_INPUT;
        }
        if (vals->arr.size() > 64) {
          set_err(err, errlen, "trace " + std::to_string(idx) + " is longer than 64 steps");
          return VFB_BAD_INPUT;
        }
        if (v == 0) o->lengths[idx] = (int)vals->arr.size();
        uint64_t w = 0;
        for (size_t t = 0; t < vals->arr.size(); ++t) {
          const JVal& x = vals->arr[t];
          const bool one = (x.kind == JVal::NUM && x.num != 0) || (x.kind == JVal::BOOL && x.b);
          if (one) w |= 1ULL << t;
        }
        o->words[(size_t)idx * nvar + v] = w;
      }
      ++idx;
    }
  }
  for (auto& s : o->names) o->name_ptrs.push_back(&s[0]);
  vfb_json_problem& pub = *o;
  pub.inst.num_vars = (int)nvar;
  pub.inst.num_traces = (int)ntr;
  pub.inst.num_pos = (int)npos;
  pub.inst.words = o->words.data();
  pub.inst.lengths = o->lengths.data();
  pub.inst.max_size = VFB_MAX_SIZE;
  pub.inst.rlx_type = 3;
  pub.max_length_traces = (int)maxlen;
  pub.names = o->name_ptrs.data();
  *out = o.release();
  return VFB_OK;
}

void vfb_json_free(vfb_json_problem* p) { delete static_cast<Owned*>(p); }

int vfb_format_infix(const vfb_result* r, const char* const* names, char* buf, size_t buflen) {
  if (!r) return -1;
  std::vector<std::string> st;
  static const char kOps[] = "~&|XFGU";
  for (int i = 0; i < r->rpn_len; ++i) {
    const int tk = r->rpn[i];
    if (tk >= 0) {
      st.push_back(names ? std::string(names[tk]) : ("p" + std::to_string(tk)));
      continue;
    }
    const int op = -tk - 1;
    if (op < 0 || op > 6) return -1;
    const char c = kOps[op];
    if (op == 0 || op == 3 || op == 4 || op == 5) {
      if (st.empty()) return -1;
      st.back() = std::string(1, c) + "(" + st.back() + ")";
    } else {
      if (st.size() < 2) return -1;
      std::string rhs = std::move(st.back());
      st.pop_back();
      st.back() = "(" + st.back() + ") " + c + " (" + rhs + ")";
    }
  }
  if (st.size() != 1) return -1;
  if (buf && buflen) std::snprintf(buf, buflen, "%s", st[0].c_str());
  return (int)st[0].size();
}

}  // extern "C"
