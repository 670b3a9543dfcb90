// Database::sql for the relational hot path: a small SQL front end and a
// planner that maps each query shape onto the GPU operators, in the fixed
// operator order of FalconDB's execute_plan (src/db.rs:1410-1416: scan+WHERE ->
// joins -> GROUP BY -> ORDER BY(+LIMIT) -> LIMIT -> projection -> DISTINCT).
//
// Supported shapes (everything else fails with FDB_E_SQL):
//   SELECT [DISTINCT] <items> FROM t [[INNER] | LEFT [OUTER]] JOIN u ON t.k = u.k]
//          [WHERE <pred>] [GROUP BY col] [ORDER BY col|alias [ASC|DESC]
//          [NULLS FIRST|LAST], ...] [LIMIT n]
//   items: *, col, COUNT(*), COUNT(col), COUNT(DISTINCT col), SUM/AVG/MIN/MAX(col),
//          ROW_NUMBER() OVER ([ORDER BY col [ASC|DESC]]) [AS a]
//   pred : col op literal, literal op col, col IS [NOT] NULL, col [NOT] IN (...),
//          col [NOT] LIKE 'pattern' (Utf8), AND, OR, parentheses, and
//          [NOT] EXISTS (SELECT ... FROM u WHERE u.k = t.k) as the whole WHERE
//          (rewritten to a SEMI / ANTI join as db.rs:1582-1604 does).
// Fast paths kept from execute_plan: COUNT(*) + WHERE counts the mask
// (db.rs:1439-1476); aggregate-only queries scan once (db.rs:1483-1518);
// ORDER BY col LIMIT k takes the bounded top-k (sort.rs:59-115); ORDER BY one
// numeric column otherwise runs the GPU radix sort.  SELECT DISTINCT takes one
// column and keeps each value's first row in output order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <set>
#include <sstream>
#include <unordered_map>

#include "engine.h"
#include "result.h"

namespace fdb {

// ===========================================================================
// Tokens
// ===========================================================================
enum TokKind { T_IDENT, T_NUM, T_STR, T_SYM, T_END };
struct Tok {
  TokKind kind;
  std::string text;   // identifiers upper-cased in `up`, symbols verbatim
  std::string up;
};

static std::vector<Tok> tokenize(const std::string& s) {
  std::vector<Tok> out;
  size_t i = 0;
  while (i < s.size()) {
    const char ch = s[i];
    if (std::isspace((unsigned char)ch)) { ++i; continue; }
    if (std::isalpha((unsigned char)ch) || ch == '_') {
      size_t j = i;
      while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
      Tok t{T_IDENT, s.substr(i, j - i), ""};
      t.up = t.text;
      for (auto& c : t.up) c = (char)std::toupper((unsigned char)c);
      out.push_back(t);
      i = j;
    } else if (ch == '"') {
      size_t j = s.find('"', i + 1);
      if (j == std::string::npos) fail(FDB_E_SQL, "unterminated quoted identifier");
      Tok t{T_IDENT, s.substr(i + 1, j - i - 1), ""};
      t.up = t.text;
      for (auto& c : t.up) c = (char)std::toupper((unsigned char)c);
      out.push_back(t);
      i = j + 1;
    } else if (std::isdigit((unsigned char)ch) || (ch == '.' && i + 1 < s.size() && std::isdigit((unsigned char)s[i + 1]))) {
      size_t j = i;
      while (j < s.size() && (std::isdigit((unsigned char)s[j]) || s[j] == '.' || s[j] == 'e' || s[j] == 'E' ||
                              ((s[j] == '+' || s[j] == '-') && (s[j - 1] == 'e' || s[j - 1] == 'E'))))
        ++j;
      out.push_back(Tok{T_NUM, s.substr(i, j - i), ""});
      i = j;
    } else if (ch == '\'') {
      std::string v;
      size_t j = i + 1;
      for (;;) {
        if (j >= s.size()) fail(FDB_E_SQL, "unterminated string literal");
        if (s[j] == '\'') {
          if (j + 1 < s.size() && s[j + 1] == '\'') { v += '\''; j += 2; continue; }
          break;
        }
        v += s[j++];
      }
      out.push_back(Tok{T_STR, v, ""});
      i = j + 1;
    } else {
      static const char* two[] = {"<>", "!=", "<=", ">="};
      bool done = false;
      for (const char* t2 : two)
        if (s.compare(i, 2, t2) == 0) {
          out.push_back(Tok{T_SYM, t2, t2});
          i += 2;
          done = true;
          break;
        }
      if (done) continue;
      if (std::strchr("(),.*=<>;-+", ch)) {
        out.push_back(Tok{T_SYM, std::string(1, ch), std::string(1, ch)});
        ++i;
      } else {
        fail(FDB_E_SQL, std::string("unexpected character '") + ch + "'");
      }
    }
  }
  out.push_back(Tok{T_END, "", ""});
  return out;
}

// ===========================================================================
// AST
// ===========================================================================
struct ColRef {
  std::string table;  // qualifier as written (may be empty)
  std::string col;
};
struct Lit {
  int kind = 0;       // FDB_INT64 | FDB_FLOAT64 | FDB_UTF8 | 0 = NULL
  int64_t i = 0;
  double f = 0.0;
  std::string s;
};
enum PredKind { P_CMP, P_ISNULL, P_NOTNULL, P_IN, P_NOTIN, P_LIKE, P_NOTLIKE, P_AND, P_OR, P_EXISTS, P_NOTEXISTS };
struct Pred {
  PredKind kind;
  ColRef col;
  int op = FDB_EQ;
  Lit lit;
  std::vector<Lit> list;
  std::unique_ptr<Pred> l, r;
  // EXISTS (SELECT .. FROM sub_table WHERE a = b)
  std::string sub_table, sub_alias;
  ColRef sub_a, sub_b;
};
struct OrderItem {
  ColRef ref;
  bool desc = false;
  bool nulls_last = false;
};
struct SelItem {
  bool star = false;
  int agg = -1;        // FDB_AGG_* or -1
  bool distinct = false;
  bool row_number = false;  // ROW_NUMBER() OVER ([ORDER BY worder])
  bool has_worder = false;
  OrderItem worder;
  ColRef col;          // empty col for COUNT(*)
  std::string alias;
  std::string text;    // default output name
};
struct Query {
  std::vector<SelItem> items;
  std::string table, alias;
  bool has_join = false;
  int join_type = FDB_JOIN_INNER;
  std::string jtable, jalias;
  ColRef on_a, on_b;
  std::unique_ptr<Pred> where;
  bool has_group = false;
  ColRef group;
  std::vector<OrderItem> order;
  int64_t limit = -1;
  bool distinct = false;  // SELECT DISTINCT (applied after ORDER BY and LIMIT, db.rs:1699-1729)
};

// ===========================================================================
// Parser
// ===========================================================================
struct Parser {
  std::vector<Tok> t;
  size_t p = 0;
  explicit Parser(const std::string& s) : t(tokenize(s)) {}
  const Tok& peek(size_t k = 0) const { return t[std::min(p + k, t.size() - 1)]; }
  bool kw(const char* w) const { return peek().kind == T_IDENT && peek().up == w; }
  bool sym(const char* s) const { return peek().kind == T_SYM && peek().text == s; }
  bool accept_kw(const char* w) {
    if (kw(w)) { ++p; return true; }
    return false;
  }
  bool accept_sym(const char* s) {
    if (sym(s)) { ++p; return true; }
    return false;
  }
  void expect_kw(const char* w) {
    if (!accept_kw(w)) fail(FDB_E_SQL, std::string("expected ") + w + " near '" + peek().text + "'");
  }
  void expect_sym(const char* s) {
    if (!accept_sym(s)) fail(FDB_E_SQL, std::string("expected '") + s + "' near '" + peek().text + "'");
  }
  static bool reserved(const std::string& up) {
    static const std::set<std::string> r = {"SELECT", "FROM",  "WHERE", "GROUP", "ORDER", "BY",    "LIMIT",
                                            "JOIN",   "INNER", "LEFT",  "OUTER", "ON",    "AND",   "OR",
                                            "NOT",    "AS",    "ASC",   "DESC",  "NULLS", "IN",    "IS",
                                            "NULL",   "LIKE",  "EXISTS", "DISTINCT"};
    return r.count(up) != 0;
  }
  std::string ident() {
    if (peek().kind != T_IDENT) fail(FDB_E_SQL, "expected an identifier near '" + peek().text + "'");
    return t[p++].text;
  }
  ColRef colref() {
    ColRef c;
    c.col = ident();
    if (accept_sym(".")) {
      c.table = c.col;
      c.col = ident();
    }
    return c;
  }
  Lit literal() {
    Lit l;
    bool neg = false;
    if (accept_sym("-")) neg = true;
    else accept_sym("+");
    const Tok& tk = peek();
    if (tk.kind == T_NUM) {
      ++p;
      const bool is_float = tk.text.find_first_of(".eE") != std::string::npos;
      if (is_float) {
        l.kind = FDB_FLOAT64;
        l.f = std::strtod(tk.text.c_str(), nullptr);
        if (neg) l.f = -l.f;
      } else {
        l.kind = FDB_INT64;
        errno = 0;
        unsigned long long v = std::strtoull(tk.text.c_str(), nullptr, 10);
        if (errno || v > (unsigned long long)INT64_MAX + (neg ? 1ull : 0ull)) {
          l.kind = FDB_FLOAT64;
          l.f = std::strtod(tk.text.c_str(), nullptr);
          if (neg) l.f = -l.f;
        } else {
          l.i = neg ? (int64_t)(0ull - v) : (int64_t)v;
        }
      }
      return l;
    }
    if (neg) fail(FDB_E_SQL, "expected a number after '-'");
    if (tk.kind == T_STR) {
      ++p;
      l.kind = FDB_UTF8;
      l.s = tk.text;
      return l;
    }
    if (kw("NULL")) {
      ++p;
      l.kind = 0;
      return l;
    }
    if (kw("TRUE") || kw("FALSE")) {
      l.kind = FDB_INT64;
      l.i = kw("TRUE") ? 1 : 0;
      ++p;
      return l;
    }
    fail(FDB_E_SQL, "expected a literal near '" + tk.text + "'");
  }
  bool at_literal() const {
    const Tok& tk = peek();
    return tk.kind == T_NUM || tk.kind == T_STR || (tk.kind == T_SYM && (tk.text == "-" || tk.text == "+")) ||
           (tk.kind == T_IDENT && (tk.up == "NULL" || tk.up == "TRUE" || tk.up == "FALSE"));
  }
  static int cmp_of(const std::string& s) {
    if (s == "=") return FDB_EQ;
    if (s == "<>" || s == "!=") return FDB_NE;
    if (s == "<") return FDB_LT;
    if (s == "<=") return FDB_LE;
    if (s == ">") return FDB_GT;
    if (s == ">=") return FDB_GE;
    return -1;
  }
  static int flip(int op) {
    switch (op) {
      case FDB_LT: return FDB_GT;
      case FDB_LE: return FDB_GE;
      case FDB_GT: return FDB_LT;
      case FDB_GE: return FDB_LE;
      default: return op;
    }
  }

  std::unique_ptr<Pred> pred_or() {
    auto l = pred_and();
    while (accept_kw("OR")) {
      auto n = std::make_unique<Pred>();
      n->kind = P_OR;
      n->l = std::move(l);
      n->r = pred_and();
      l = std::move(n);
    }
    return l;
  }
  std::unique_ptr<Pred> pred_and() {
    auto l = pred_prim();
    while (accept_kw("AND")) {
      auto n = std::make_unique<Pred>();
      n->kind = P_AND;
      n->l = std::move(l);
      n->r = pred_prim();
      l = std::move(n);
    }
    return l;
  }
  std::unique_ptr<Pred> pred_prim() {
    if (sym("(")) {
      // Parenthesised predicate (a sub-SELECT only appears after EXISTS).
      ++p;
      auto e = pred_or();
      expect_sym(")");
      return e;
    }
    if (kw("NOT") && peek(1).kind == T_IDENT && peek(1).up == "EXISTS") {
      p += 2;
      auto e = exists_body();
      e->kind = P_NOTEXISTS;
      return e;
    }
    if (accept_kw("EXISTS")) {
      auto e = exists_body();
      e->kind = P_EXISTS;
      return e;
    }
    auto n = std::make_unique<Pred>();
    if (at_literal()) {
      // literal op col
      Lit l = literal();
      const int op = cmp_of(peek().text);
      if (peek().kind != T_SYM || op < 0) fail(FDB_E_SQL, "expected a comparison");
      ++p;
      n->kind = P_CMP;
      n->col = colref();
      n->op = flip(op);
      n->lit = l;
      return n;
    }
    n->col = colref();
    if (accept_kw("IS")) {
      const bool neg = accept_kw("NOT");
      expect_kw("NULL");
      n->kind = neg ? P_NOTNULL : P_ISNULL;
      return n;
    }
    bool neg = accept_kw("NOT");
    if (accept_kw("IN")) {
      n->kind = neg ? P_NOTIN : P_IN;
      expect_sym("(");
      do {
        n->list.push_back(literal());
      } while (accept_sym(","));
      expect_sym(")");
      return n;
    }
    if (accept_kw("LIKE")) {
      n->kind = neg ? P_NOTLIKE : P_LIKE;
      n->lit = literal();
      if (n->lit.kind != FDB_UTF8) fail(FDB_E_SQL, "LIKE needs a string pattern");
      return n;
    }
    if (neg) fail(FDB_E_SQL, "expected IN or LIKE after NOT");
    const int op = cmp_of(peek().text);
    if (peek().kind != T_SYM || op < 0) fail(FDB_E_SQL, "expected a comparison near '" + peek().text + "'");
    ++p;
    n->kind = P_CMP;
    n->op = op;
    n->lit = literal();
    return n;
  }
  std::unique_ptr<Pred> exists_body() {
    // ( SELECT <anything> FROM u [alias] WHERE a = b )
    auto e = std::make_unique<Pred>();
    expect_sym("(");
    expect_kw("SELECT");
    int depth = 0;
    while (!(depth == 0 && kw("FROM"))) {
      if (peek().kind == T_END) fail(FDB_E_SQL, "unterminated EXISTS subquery");
      if (sym("(")) ++depth;
      if (sym(")")) --depth;
      ++p;
    }
    expect_kw("FROM");
    e->sub_table = ident();
    if (accept_kw("AS")) e->sub_alias = ident();
    else if (peek().kind == T_IDENT && !reserved(peek().up)) e->sub_alias = ident();
    expect_kw("WHERE");
    e->sub_a = colref();
    expect_sym("=");
    e->sub_b = colref();
    if (!sym(")")) fail(FDB_E_SQL, "EXISTS subquery supports exactly one equality");
    expect_sym(")");
    return e;
  }

  SelItem sel_item() {
    SelItem it;
    if (accept_sym("*")) {
      it.star = true;
      it.text = "*";
      return it;
    }
    if (peek().kind == T_IDENT && peek().up == "ROW_NUMBER" && peek(1).kind == T_SYM && peek(1).text == "(") {
      // ROW_NUMBER() OVER ([ORDER BY col [ASC|DESC]]) (window.rs:97-260)
      p += 2;
      expect_sym(")");
      if (!(peek().kind == T_IDENT && peek().up == "OVER")) fail(FDB_E_SQL, "ROW_NUMBER() needs OVER (...)");
      ++p;
      expect_sym("(");
      if (peek().kind == T_IDENT && peek().up == "PARTITION")
        fail(FDB_E_SQL, "ROW_NUMBER() OVER (PARTITION BY ..) is not supported");
      it.row_number = true;
      it.text = "ROW_NUMBER()";
      if (accept_kw("ORDER")) {
        expect_kw("BY");
        it.has_worder = true;
        it.worder.ref = colref();
        if (accept_kw("DESC")) it.worder.desc = true;
        else accept_kw("ASC");
        if (sym(",")) fail(FDB_E_SQL, "ROW_NUMBER() OVER (ORDER BY ..) takes one key");
      }
      expect_sym(")");
      if (accept_kw("AS")) it.alias = ident();
      else if (peek().kind == T_IDENT && !reserved(peek().up)) it.alias = ident();
      return it;
    }
    static const std::pair<const char*, int> aggs[] = {{"COUNT", FDB_AGG_COUNT}, {"SUM", FDB_AGG_SUM},
                                                        {"AVG", FDB_AGG_AVG},     {"MIN", FDB_AGG_MIN},
                                                        {"MAX", FDB_AGG_MAX}};
    if (peek().kind == T_IDENT && peek(1).kind == T_SYM && peek(1).text == "(") {
      int agg = -1;
      for (auto& a : aggs)
        if (peek().up == a.first) agg = a.second;
      if (agg < 0) fail(FDB_E_SQL, "unsupported function " + peek().text);
      const std::string fname = peek().up;
      p += 2;
      if (agg == FDB_AGG_COUNT && accept_sym("*")) {
        it.agg = FDB_AGG_COUNT_STAR;
        it.text = "COUNT(*)";
      } else {
        if (accept_kw("DISTINCT")) {
          if (agg != FDB_AGG_COUNT) fail(FDB_E_SQL, "DISTINCT is supported in COUNT only");
          it.distinct = true;
          agg = FDB_AGG_COUNT_DISTINCT;
        }
        if (at_literal()) {
          Lit l = literal();
          if (agg == FDB_AGG_COUNT && l.kind != 0) {
            agg = FDB_AGG_COUNT_STAR;  // COUNT(1) counts rows (sql.rs:884-885)
          } else {
            fail(FDB_E_SQL, "aggregate over a literal is not supported");
          }
          it.text = "COUNT(*)";
        } else {
          it.col = colref();
          it.text = fname + "(" + (it.distinct ? "DISTINCT " : "") + it.col.col + ")";
        }
        it.agg = agg;
      }
      expect_sym(")");
    } else {
      it.col = colref();
      it.text = it.col.col;
    }
    if (accept_kw("AS")) it.alias = ident();
    else if (peek().kind == T_IDENT && !reserved(peek().up)) it.alias = ident();
    return it;
  }

  Query query() {
    Query q;
    expect_kw("SELECT");
    if (accept_kw("DISTINCT")) q.distinct = true;
    do {
      q.items.push_back(sel_item());
    } while (accept_sym(","));
    expect_kw("FROM");
    q.table = ident();
    if (accept_kw("AS")) q.alias = ident();
    else if (peek().kind == T_IDENT && !reserved(peek().up)) q.alias = ident();
    if (kw("JOIN") || kw("INNER") || kw("LEFT")) {
      q.has_join = true;
      if (accept_kw("LEFT")) {
        accept_kw("OUTER");
        q.join_type = FDB_JOIN_LEFT;
      } else {
        accept_kw("INNER");
        q.join_type = FDB_JOIN_INNER;
      }
      expect_kw("JOIN");
      q.jtable = ident();
      if (accept_kw("AS")) q.jalias = ident();
      else if (peek().kind == T_IDENT && !reserved(peek().up)) q.jalias = ident();
      expect_kw("ON");
      q.on_a = colref();
      expect_sym("=");
      q.on_b = colref();
    }
    if (accept_kw("WHERE")) q.where = pred_or();
    if (accept_kw("GROUP")) {
      expect_kw("BY");
      q.has_group = true;
      q.group = colref();
      if (sym(",")) fail(FDB_E_SQL, "GROUP BY supports one key column");
    }
    if (accept_kw("ORDER")) {
      expect_kw("BY");
      do {
        OrderItem o;
        if (peek().kind == T_NUM) {
          o.ref.col = "#" + peek().text;  // ordinal
          ++p;
        } else {
          o.ref = colref();
        }
        if (accept_kw("DESC")) o.desc = true;
        else accept_kw("ASC");
        o.nulls_last = o.desc;  // sql.rs:1486-1491 defaults
        if (accept_kw("NULLS")) {
          if (accept_kw("FIRST")) o.nulls_last = false;
          else if (accept_kw("LAST")) o.nulls_last = true;
          else fail(FDB_E_SQL, "expected FIRST or LAST after NULLS");
        }
        q.order.push_back(o);
      } while (accept_sym(","));
    }
    if (accept_kw("LIMIT")) {
      Lit l = literal();
      if (l.kind != FDB_INT64 || l.i < 0) fail(FDB_E_SQL, "LIMIT needs a non-negative integer");
      q.limit = l.i;
    }
    accept_sym(";");
    if (peek().kind != T_END) fail(FDB_E_SQL, "unexpected '" + peek().text + "' at the end of the query");
    return q;
  }
};

// ===========================================================================
// Planner / executor
// ===========================================================================

// A device-resident relation the plan reads: either a catalog table or a
// temporary one (the materialised output of a join).
struct RelCol {
  std::string name;     // bare column name
  std::string qual;     // table name or alias it belongs to
  std::string qual2;    // the other spelling (alias <-> table name)
  int32_t dtype = 0;
  fdb_dev_column dev{};
  const std::vector<std::string>* dict = nullptr;
  Column* src = nullptr;  // the catalog column (zone maps), for a catalog table
};
struct Rel {
  uint64_t nrows = 0;
  std::vector<RelCol> cols;
  std::vector<DevBuf> owned;  // temporary buffers (freed with the plan)
};

struct Plan {
  Ctx& c;
  std::vector<DevBuf> bufs;   // per-query device buffers
  explicit Plan(Ctx& ctx) : c(ctx) {}
  ~Plan() {
    cudaStreamSynchronize(c.stream);
    for (auto& b : bufs) c.free_buf(b);
  }
  template <typename T>
  T* dev(size_t n) {
    bufs.push_back(c.alloc_buf(std::max<size_t>(n, 1) * sizeof(T)));
    return static_cast<T*>(bufs.back().ptr);
  }
  template <typename T>
  std::vector<T> to_host(const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) FDB_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    FDB_CUDA(cudaStreamSynchronize(c.stream));
    return h;
  }
  template <typename T>
  T one(const T* d) {
    return to_host(d, 1)[0];
  }
  void check() {
    const int e = c.check_device_error();
    if (e) fail(e, e == FDB_E_TIMEOUT ? "a device-side wait timed out" : "an operator output overflowed");
  }
};

static void add_table_cols(Ctx& c, Rel& r, Table& t, const std::string& alias) {
  r.nrows = t.nrows;
  for (Column& col : t.cols) {
    RelCol rc;
    rc.name = col.name;
    rc.qual = alias.empty() ? t.name : alias;
    rc.qual2 = t.name;
    rc.dtype = col.dtype;
    rc.dev.dtype = col.dtype;
    rc.dev.values = col.values.ptr;
    rc.dev.validity = static_cast<const uint64_t*>(col.validity.ptr);
    rc.dev.validity_offset = 0;
    rc.dict = &col.dict;
    rc.src = &col;
    FDB_CUDA(cudaStreamWaitEvent(c.stream, col.ready, 0));
    r.cols.push_back(rc);
  }
}

static int resolve(const Rel& r, const ColRef& ref) {
  int found = -1;
  for (size_t i = 0; i < r.cols.size(); ++i) {
    const RelCol& rc = r.cols[i];
    if (rc.name != ref.col) continue;
    if (!ref.table.empty() && rc.qual != ref.table && rc.qual2 != ref.table) continue;
    if (found >= 0) fail(FDB_E_SQL, "ambiguous column " + ref.col);
    found = (int)i;
  }
  if (found < 0) fail(FDB_E_NOTFOUND, "no column " + (ref.table.empty() ? "" : ref.table + ".") + ref.col);
  return found;
}

static std::shared_ptr<Table> find_table(Ctx& c, const std::string& name) {
  auto it = c.tables.find(name);
  if (it == c.tables.end()) fail(FDB_E_NOTFOUND, "no table " + name);
  return it->second;
}

// SQL LIKE with % and _ over bytes.
static bool like_match(const std::string& s, const std::string& p) {
  size_t si = 0, pi = 0, star = std::string::npos, mark = 0;
  while (si < s.size()) {
    if (pi < p.size() && (p[pi] == '_' || p[pi] == s[si])) { ++si; ++pi; }
    else if (pi < p.size() && p[pi] == '%') { star = pi++; mark = si; }
    else if (star != std::string::npos) { pi = star + 1; si = ++mark; }
    else return false;
  }
  while (pi < p.size() && p[pi] == '%') ++pi;
  return pi == p.size();
}

// Compiles a WHERE tree into postfix terms over a local column list.
struct PredCompiler {
  Plan& plan;
  const Rel& rel;
  std::vector<int>& local;           // local column index -> rel column
  std::vector<fdb_pred_term> terms;
  std::vector<std::vector<uint64_t>> host_sets;  // per term: the CODE_SET bitmap on the host

  int local_of(int relcol) {
    for (size_t i = 0; i < local.size(); ++i)
      if (local[i] == relcol) return (int)i;
    local.push_back(relcol);
    return (int)local.size() - 1;
  }
  void push_false(int col) {
    // A leaf that never passes: IS NULL AND IS NOT NULL.
    fdb_pred_term a{}, b{}, n{};
    a.kind = FDB_TERM_IS_NULL;
    a.col = col;
    b.kind = FDB_TERM_IS_NOT_NULL;
    b.col = col;
    n.kind = FDB_TERM_AND;
    terms.push_back(a);
    terms.push_back(b);
    terms.push_back(n);
  }
  void code_set(int col, const std::vector<bool>& pass) {
    const size_t words = std::max<size_t>(1, (pass.size() + 63) / 64);
    std::vector<uint64_t> bits(words, 0);
    for (size_t i = 0; i < pass.size(); ++i)
      if (pass[i]) bits[i >> 6] |= 1ull << (i & 63);
    uint64_t* d = plan.dev<uint64_t>(words);
    FDB_CUDA(cudaMemcpyAsync(d, bits.data(), words * 8, cudaMemcpyHostToDevice, plan.c.stream));
    FDB_CUDA(cudaStreamSynchronize(plan.c.stream));
    fdb_pred_term t{};
    t.kind = FDB_TERM_CODE_SET;
    t.col = col;
    t.lit_i = (int64_t)pass.size();
    t.code_set = d;
    host_sets.resize(terms.size());
    host_sets.push_back(std::move(bits));
    terms.push_back(t);
  }
  void leaf_cmp(int rc, int lc, int op, const Lit& lit) {
    const RelCol& col = rel.cols[rc];
    if (lit.kind == 0) {  // comparison with NULL never passes
      push_false(lc);
      return;
    }
    if (col.dtype == FDB_UTF8) {
      if (lit.kind != FDB_UTF8) fail(FDB_E_TYPE, "comparing text column " + col.name + " with a number");
      std::vector<bool> pass(col.dict->size());
      for (size_t i = 0; i < pass.size(); ++i) {
        const int c = (*col.dict)[i].compare(lit.s);
        switch (op) {
          case FDB_EQ: pass[i] = c == 0; break;
          case FDB_NE: pass[i] = c != 0; break;
          case FDB_LT: pass[i] = c < 0; break;
          case FDB_LE: pass[i] = c <= 0; break;
          case FDB_GT: pass[i] = c > 0; break;
          default: pass[i] = c >= 0; break;
        }
      }
      code_set(lc, pass);
      return;
    }
    if (lit.kind == FDB_UTF8) fail(FDB_E_TYPE, "comparing numeric column " + col.name + " with text");
    fdb_pred_term t{};
    t.kind = FDB_TERM_CMP;
    t.col = lc;
    t.op = op;
    t.lit_type = lit.kind;
    t.lit_i = lit.i;
    t.lit_f = lit.f;
    terms.push_back(t);
  }
  void join(int kind) {
    fdb_pred_term t{};
    t.kind = kind;
    terms.push_back(t);
  }
  void compile(const Pred& p) {
    switch (p.kind) {
      case P_AND:
      case P_OR:
        compile(*p.l);
        compile(*p.r);
        join(p.kind == P_AND ? FDB_TERM_AND : FDB_TERM_OR);
        return;
      case P_EXISTS:
      case P_NOTEXISTS:
        fail(FDB_E_SQL, "EXISTS must be the whole WHERE clause");
      default: break;
    }
    const int rc = resolve(rel, p.col);
    const int lc = local_of(rc);
    const RelCol& col = rel.cols[rc];
    switch (p.kind) {
      case P_CMP: leaf_cmp(rc, lc, p.op, p.lit); break;
      case P_ISNULL:
      case P_NOTNULL: {
        fdb_pred_term t{};
        t.kind = p.kind == P_ISNULL ? FDB_TERM_IS_NULL : FDB_TERM_IS_NOT_NULL;
        t.col = lc;
        terms.push_back(t);
        break;
      }
      case P_IN:
      case P_NOTIN: {
        if (col.dtype == FDB_UTF8) {
          std::vector<bool> pass(col.dict->size(), p.kind == P_NOTIN);
          for (size_t i = 0; i < pass.size(); ++i)
            for (const Lit& l : p.list)
              if (l.kind == FDB_UTF8 && (*col.dict)[i] == l.s) pass[i] = p.kind == P_IN;
          code_set(lc, pass);
          break;
        }
        // numeric: OR of EQ (IN) / AND of NE (NOT IN); NULL rows fail both.
        // A NULL in the list matches nothing for IN and makes NOT IN never
        // true (SQL three-valued logic).
        bool first = true;
        for (const Lit& l : p.list) {
          if (l.kind == 0) {
            if (p.kind == P_IN) continue;
            push_false(lc);
          } else {
            leaf_cmp(rc, lc, p.kind == P_IN ? FDB_EQ : FDB_NE, l);
          }
          if (!first) join(p.kind == P_IN ? FDB_TERM_OR : FDB_TERM_AND);
          first = false;
        }
        if (first) push_false(lc);
        break;
      }
      case P_LIKE:
      case P_NOTLIKE: {
        if (col.dtype != FDB_UTF8) fail(FDB_E_TYPE, "LIKE needs a text column");
        std::vector<bool> pass(col.dict->size());
        for (size_t i = 0; i < pass.size(); ++i) {
          const bool m = like_match((*col.dict)[i], p.lit.s);
          pass[i] = p.kind == P_LIKE ? m : !m;
        }
        code_set(lc, pass);
        break;
      }
      default: fail(FDB_E_SQL, "unsupported predicate");
    }
    if (terms.size() > FDB_MAX_TERMS) fail(FDB_E_SQL, "WHERE clause too long for one scan");
  }
};

static std::vector<fdb_dev_column> local_cols(const Rel& r, const std::vector<int>& local) {
  std::vector<fdb_dev_column> v;
  for (int i : local) v.push_back(r.cols[i].dev);
  return v;
}

// Host-side output builder.
static void push_col(fdb_result* res, const std::string& name, int dtype) {
  fdb_result::Col c;
  c.name = name;
  c.dtype = dtype;
  res->cols.push_back(std::move(c));
}

// Fetch rows `rows` (host list) of rel column rc into a result column.
static void fetch_rows(Plan& plan, const Rel& r, int rc, const uint32_t* d_rows, uint64_t n,
                       fdb_result::Col& out) {
  const RelCol& col = r.cols[rc];
  const int esz = dtype_size(col.dtype);
  void* d_vals = plan.dev<uint8_t>(n * esz);
  uint64_t* d_valid = nullptr;
  if (col.dev.validity) d_valid = plan.dev<uint64_t>((n + 63) / 64);
  op_gather(plan.c, col.dev, d_rows, n, d_vals, d_valid);
  std::vector<uint8_t> raw = plan.to_host(static_cast<uint8_t*>(d_vals), n * esz);
  std::vector<uint64_t> vw;
  if (d_valid) vw = plan.to_host(d_valid, (n + 63) / 64);
  out.nulls.assign(n, 0);
  if (col.dtype == FDB_INT64 || col.dtype == FDB_FLOAT64) {
    if (col.dtype == FDB_INT64) {
      out.i64.resize(n);
      if (n) std::memcpy(out.i64.data(), raw.data(), n * 8);
    } else {
      out.f64.resize(n);
      if (n) std::memcpy(out.f64.data(), raw.data(), n * 8);
    }
    if (!vw.empty())
      for (uint64_t i = 0; i < n; ++i) out.nulls[i] = ((vw[i >> 6] >> (i & 63)) & 1ull) ? 0 : 1;
    return;
  }
  out.str.reserve(n);
  for (uint64_t i = 0; i < n; ++i) {  // UTF8: codes to strings
    const bool valid = vw.empty() || ((vw[i >> 6] >> (i & 63)) & 1ull);
    uint32_t code;
    std::memcpy(&code, raw.data() + i * 4, 4);
    const bool ok = valid && code != 0xFFFFFFFFu && code < col.dict->size();
    out.str.push_back(ok ? (*col.dict)[code] : std::string());
    if (!ok) out.nulls[i] = 1;
  }
}

// The rank of every code of a text column's dictionary in the sorted
// dictionary, on the device: byte-wise string order (Rust's str ordering,
// which the reference's text sort uses, sort.rs:352-382); equal strings under
// two codes get one rank.  The dictionary holds distinct strings, not rows, so
// ranking it on the host is cheap; the rows are then sorted on the GPU.
static const uint32_t* dict_ranks(Plan& plan, const RelCol& col) {
  const std::vector<std::string>& d = *col.dict;
  std::vector<uint32_t> idx(d.size());
  std::iota(idx.begin(), idx.end(), 0u);
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return d[a] < d[b]; });
  std::vector<uint32_t> rank(std::max<size_t>(d.size(), 1), 0);
  for (size_t i = 0; i < idx.size(); ++i)
    rank[idx[i]] = (i > 0 && d[idx[i]] == d[idx[i - 1]]) ? rank[idx[i - 1]] : (uint32_t)i;
  uint32_t* dr = plan.dev<uint32_t>(rank.size());
  // From pageable memory: the call returns once the source has been staged.
  FDB_CUDA(cudaMemcpyAsync(dr, rank.data(), rank.size() * 4, cudaMemcpyHostToDevice, plan.c.stream));
  return dr;
}

// ---------------------------------------------------------------------------
// Scalar value model used for ORDER BY over host results.
// ---------------------------------------------------------------------------
static int cmp_cell(const fdb_result::Col& c, uint64_t a, uint64_t b) {
  const bool na = !c.nulls.empty() && c.nulls[a], nb = !c.nulls.empty() && c.nulls[b];
  if (na || nb) return na == nb ? 0 : (na ? -2 : 2);  // +-2 marks NULL involvement
  if (c.dtype == FDB_INT64) return c.i64[a] < c.i64[b] ? -1 : c.i64[a] > c.i64[b] ? 1 : 0;
  if (c.dtype == FDB_FLOAT64) {
    const double x = c.f64[a], y = c.f64[b];
    if (std::isnan(x) || std::isnan(y)) return std::isnan(x) == std::isnan(y) ? 0 : (std::isnan(x) ? 1 : -1);
    return x < y ? -1 : x > y ? 1 : 0;
  }
  return c.str[a].compare(c.str[b]) < 0 ? -1 : (c.str[a] == c.str[b] ? 0 : 1);
}

static void apply_order_limit(fdb_result* res, const std::vector<std::pair<int, OrderItem>>& keys, int64_t limit) {
  std::vector<uint64_t> idx(res->rows);
  std::iota(idx.begin(), idx.end(), 0);
  if (!keys.empty()) {
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
      for (auto& k : keys) {
        const int c = cmp_cell(res->cols[k.first], a, b);
        if (c == 0) continue;
        if (c == 2 || c == -2) {  // NULL vs value: a is NULL when c == -2
          const bool a_null = c == -2;
          return k.second.nulls_last ? !a_null : a_null;
        }
        return k.second.desc ? c > 0 : c < 0;
      }
      return false;
    });
  }
  if (limit >= 0 && (uint64_t)limit < idx.size()) idx.resize((size_t)limit);
  for (auto& col : res->cols) {
    fdb_result::Col n;
    n.name = col.name;
    n.dtype = col.dtype;
    for (uint64_t i : idx) {
      if (col.dtype == FDB_INT64) n.i64.push_back(col.i64[i]);
      else if (col.dtype == FDB_FLOAT64) n.f64.push_back(col.f64[i]);
      else n.str.push_back(col.str[i]);
      n.nulls.push_back(col.nulls.empty() ? 0 : col.nulls[i]);
    }
    col = std::move(n);
  }
  res->rows = idx.size();
}

static std::string out_name(const SelItem& it) { return it.alias.empty() ? it.text : it.alias; }

// ORDER BY references resolve against output names (alias / default text /
// bare column) or 1-based ordinals.
static std::vector<std::pair<int, OrderItem>> order_keys(const fdb_result* res, const Query& q,
                                                         const std::vector<SelItem>& items) {
  std::vector<std::pair<int, OrderItem>> keys;
  for (const OrderItem& o : q.order) {
    int idx = -1;
    if (!o.ref.col.empty() && o.ref.col[0] == '#') {
      idx = std::atoi(o.ref.col.c_str() + 1) - 1;
      if (idx < 0 || idx >= (int)res->cols.size()) fail(FDB_E_SQL, "ORDER BY ordinal out of range");
    } else {
      for (size_t i = 0; i < items.size() && i < res->cols.size(); ++i) {
        const SelItem& it = items[i];
        if (it.alias == o.ref.col || (it.agg < 0 && it.col.col == o.ref.col) || it.text == o.ref.col) {
          idx = (int)i;
          break;
        }
      }
      if (idx < 0)
        for (size_t i = 0; i < res->cols.size(); ++i)
          if (res->cols[i].name == o.ref.col) idx = (int)i;
    }
    if (idx < 0) fail(FDB_E_SQL, "ORDER BY " + o.ref.col + " must name an output column here");
    keys.push_back({idx, o});
  }
  return keys;
}

// ---------------------------------------------------------------------------
// Aggregates without GROUP BY (execute_agg_only, aggregate.rs:1394-1528).
// ---------------------------------------------------------------------------
static void run_aggregates(Plan& plan, const Rel& rel, const Query& q, fdb_result* res) {
  std::vector<int> local;
  PredCompiler pc{plan, rel, local, {}};
  if (q.where) pc.compile(*q.where);
  const std::vector<fdb_pred_term> prog = pc.terms;
  const size_t pred_cols = local.size();

  // COUNT(*) + WHERE alone: count the mask (db.rs:1439-1476).
  if (q.items.size() == 1 && q.items[0].agg == FDB_AGG_COUNT_STAR) {
    push_col(res, out_name(q.items[0]), FDB_INT64);
    uint64_t* d = plan.dev<uint64_t>(1);
    std::vector<fdb_dev_column> cols = local_cols(rel, local);
    if (rel.nrows == 0) {
      res->cols[0].i64.push_back(0);
    } else if (cols.empty()) {
      res->cols[0].i64.push_back((int64_t)rel.nrows);
    } else {
      op_filter_count(plan.c, cols.data(), (int)cols.size(), rel.nrows, prog.data(), (int)prog.size(), d);
      plan.check();
      res->cols[0].i64.push_back((int64_t)plan.one(d));
    }
    res->cols[0].nulls.push_back(0);
    res->rows = 1;
    return;
  }

  for (const SelItem& it : q.items) {
    if (it.agg < 0 || it.star) fail(FDB_E_SQL, "mixing aggregates and plain columns needs GROUP BY");
    push_col(res, out_name(it), (it.agg == FDB_AGG_COUNT_STAR || it.agg == FDB_AGG_COUNT ||
                                 it.agg == FDB_AGG_COUNT_DISTINCT)
                                    ? FDB_INT64
                                    : FDB_FLOAT64);
  }
  res->rows = 1;
  // Numeric aggregates in scans of up to 4 aggregates and 4 columns.
  std::vector<size_t> pending;
  for (size_t i = 0; i < q.items.size(); ++i)
    if (q.items[i].agg != FDB_AGG_COUNT_DISTINCT) pending.push_back(i);
  size_t pi = 0;
  while (pi < pending.size()) {
    std::vector<int> loc(local.begin(), local.begin() + pred_cols);
    std::vector<fdb_agg_spec> specs;
    std::vector<size_t> which;
    while (pi < pending.size() && specs.size() < 4) {
      const SelItem& it = q.items[pending[pi]];
      fdb_agg_spec s{};
      s.func = it.agg;
      s.col = 0;
      if (it.agg != FDB_AGG_COUNT_STAR) {
        const int rc = resolve(rel, it.col);
        int lc = -1;
        for (size_t k = 0; k < loc.size(); ++k)
          if (loc[k] == rc) lc = (int)k;
        if (lc < 0) {
          if (loc.size() >= 4) break;
          loc.push_back(rc);
          lc = (int)loc.size() - 1;
        }
        s.col = lc;
        if (rel.cols[rc].dtype == FDB_UTF8 && it.agg != FDB_AGG_COUNT)
          fail(FDB_E_TYPE, it.text + " needs a numeric column");
      }
      specs.push_back(s);
      which.push_back(pending[pi]);
      ++pi;
    }
    if (specs.empty()) fail(FDB_E_SQL, "too many columns in one aggregate query");
    if (loc.empty()) loc.push_back(0);  // COUNT(*) without WHERE still needs a column to scan
    std::vector<fdb_dev_column> cols = local_cols(rel, loc);
    fdb_agg_value* d = plan.dev<fdb_agg_value>(specs.size());
    if (rel.nrows == 0 || rel.cols.empty()) {
      FDB_CUDA(cudaMemsetAsync(d, 0, sizeof(fdb_agg_value) * specs.size(), plan.c.stream));
      std::vector<fdb_agg_value> h = plan.to_host(d, specs.size());
      for (size_t k = 0; k < specs.size(); ++k) {
        auto& col = res->cols[which[k]];
        if (col.dtype == FDB_INT64) { col.i64.push_back(0); col.nulls.push_back(0); }
        else { col.f64.push_back(0.0); col.nulls.push_back(1); }
      }
      continue;
    }
    op_aggregate(plan.c, cols.data(), (int)cols.size(), rel.nrows, prog.data(), (int)prog.size(), specs.data(),
                 (int)specs.size(), d);
    plan.check();
    std::vector<fdb_agg_value> h = plan.to_host(d, specs.size());
    for (size_t k = 0; k < specs.size(); ++k) {
      auto& col = res->cols[which[k]];
      if (col.dtype == FDB_INT64) {
        col.i64.push_back(h[k].i);
        col.nulls.push_back(0);
      } else {
        col.f64.push_back(h[k].f);
        col.nulls.push_back(h[k].valid ? 0 : 1);
      }
    }
  }
  // COUNT(DISTINCT col)
  for (size_t i = 0; i < q.items.size(); ++i) {
    const SelItem& it = q.items[i];
    if (it.agg != FDB_AGG_COUNT_DISTINCT) continue;
    const int rc = resolve(rel, it.col);
    const RelCol& col = rel.cols[rc];
    int64_t result = 0;
    if (rel.nrows > 0 && col.dtype == FDB_UTF8) {
      std::vector<int> loc(local.begin(), local.begin() + pred_cols);
      int lc = -1;
      for (size_t k = 0; k < loc.size(); ++k)
        if (loc[k] == rc) lc = (int)k;
      if (lc < 0) {
        loc.push_back(rc);
        lc = (int)loc.size() - 1;
      }
      std::vector<fdb_dev_column> cols = local_cols(rel, loc);
      const uint32_t dl = (uint32_t)col.dict->size();
      uint64_t* d = plan.dev<uint64_t>((dl + 63) / 64);
      op_distinct_codes(plan.c, cols.data(), (int)cols.size(), rel.nrows, prog.data(), (int)prog.size(), lc, dl, d);
      plan.check();
      std::vector<uint64_t> bits = plan.to_host(d, (dl + 63) / 64);
      std::set<std::string> seen;  // DistinctSet::Strings over the present codes
      for (uint32_t code = 0; code < dl; ++code)
        if ((bits[code >> 6] >> (code & 63)) & 1ull) seen.insert((*col.dict)[code]);
      result = (int64_t)seen.size();
    } else if (rel.nrows > 0 && col.dtype == FDB_INT64) {
      std::vector<fdb_dev_column> pcols = local_cols(rel, std::vector<int>(local.begin(), local.begin() + pred_cols));
      if (pcols.size() > 2) fail(FDB_E_SQL, "COUNT(DISTINCT) with a WHERE over more than 2 columns");
      const uint64_t cap = rel.nrows + 1;
      fdb_group_i64* d = plan.dev<fdb_group_i64>(cap);
      uint64_t* dn = plan.dev<uint64_t>(1);
      plan.c.scratch_reset();
      const GbSizing sz = group_by_i64_sizing(plan.c, col.dev, rel.nrows, 0);
      plan.c.scratch_reset();
      plan.c.ensure_scratch(group_by_i64_scratch(sz, 0.5) + (16u << 20));
      op_group_by_i64(plan.c, col.dev, col.dev, rel.nrows, prog.data(), (int)prog.size(), pcols.data(),
                      (int)pcols.size(), sz, 0.5, d, cap, dn);
      plan.check();
      const uint64_t ng = plan.one(dn);
      std::vector<fdb_group_i64> g = plan.to_host(d, ng);
      for (auto& x : g)
        if (!(x.key == INT64_MIN)) ++result;  // NULL is not a distinct value
    } else if (rel.nrows > 0) {
      fail(FDB_E_SQL, "COUNT(DISTINCT) over a FLOAT64 column is not supported");
    }
    res->cols[i].i64.push_back(result);
    res->cols[i].nulls.push_back(0);
  }
}

// ---------------------------------------------------------------------------
// GROUP BY
// ---------------------------------------------------------------------------
static void run_group_by(Plan& plan, const Rel& rel, const Query& q, fdb_result* res) {
  const int kc = resolve(rel, q.group);
  const RelCol& key = rel.cols[kc];
  std::vector<int> local;
  PredCompiler pc{plan, rel, local, {}};
  if (q.where) pc.compile(*q.where);
  const std::vector<fdb_pred_term> prog = pc.terms;
  // Output columns.
  for (const SelItem& it : q.items) {
    if (it.star) fail(FDB_E_SQL, "SELECT * with GROUP BY");
    if (it.agg < 0) {
      const int rc = resolve(rel, it.col);
      if (rc != kc) fail(FDB_E_SQL, "column " + it.col.col + " must appear in GROUP BY");
      push_col(res, out_name(it), key.dtype);
    } else {
      if (it.agg == FDB_AGG_COUNT_DISTINCT) fail(FDB_E_SQL, "COUNT(DISTINCT) inside GROUP BY is not supported");
      push_col(res, out_name(it), (it.agg == FDB_AGG_COUNT_STAR || it.agg == FDB_AGG_COUNT) ? FDB_INT64 : FDB_FLOAT64);
    }
  }
  std::vector<size_t> agg_items;
  for (size_t i = 0; i < q.items.size(); ++i)
    if (q.items[i].agg >= 0) agg_items.push_back(i);

  if (key.dtype == FDB_UTF8) {
    const uint32_t dl = (uint32_t)key.dict->size();
    const uint32_t ng = dl + 1;
    std::vector<int64_t> group_rows(ng, 0);
    std::vector<std::vector<fdb_agg_value>> vals(q.items.size());
    bool rows_known = false;
    size_t ai = 0;
    do {
      std::vector<int> loc = local;
      int klc = -1;
      for (size_t k = 0; k < loc.size(); ++k)
        if (loc[k] == kc) klc = (int)k;
      if (klc < 0) {
        loc.push_back(kc);
        klc = (int)loc.size() - 1;
      }
      std::vector<fdb_agg_spec> specs;
      std::vector<size_t> which;
      while (ai < agg_items.size() && specs.size() < 4) {
        const SelItem& it = q.items[agg_items[ai]];
        fdb_agg_spec s{};
        s.func = it.agg;
        if (it.agg != FDB_AGG_COUNT_STAR) {
          const int rc = resolve(rel, it.col);
          int lc = -1;
          for (size_t k = 0; k < loc.size(); ++k)
            if (loc[k] == rc) lc = (int)k;
          if (lc < 0) {
            if (loc.size() >= 4) break;
            loc.push_back(rc);
            lc = (int)loc.size() - 1;
          }
          s.col = lc;
        }
        specs.push_back(s);
        which.push_back(agg_items[ai]);
        ++ai;
      }
      if (specs.empty()) {
        if (ai < agg_items.size()) fail(FDB_E_SQL, "too many columns in one GROUP BY query");
        fdb_agg_spec s{};
        s.func = FDB_AGG_COUNT_STAR;
        specs.push_back(s);
      }
      std::vector<fdb_dev_column> cols = local_cols(rel, loc);
      fdb_agg_value* d = plan.dev<fdb_agg_value>((size_t)ng * specs.size());
      int64_t* dr = plan.dev<int64_t>(ng);
      if (rel.nrows > 0) {
        op_group_by_codes(plan.c, cols.data(), (int)cols.size(), rel.nrows, prog.data(), (int)prog.size(), klc, dl,
                          specs.data(), (int)specs.size(), d, dr);
        plan.check();
        std::vector<fdb_agg_value> h = plan.to_host(d, (size_t)ng * specs.size());
        if (!rows_known) {
          group_rows = plan.to_host(dr, ng);
          rows_known = true;
        }
        for (size_t k = 0; k < which.size(); ++k) {
          vals[which[k]].resize(ng);
          for (uint32_t g = 0; g < ng; ++g) vals[which[k]][g] = h[(size_t)g * specs.size() + k];
        }
      }
    } while (ai < agg_items.size());
    // Emit present groups in dictionary order (ORDER BY below fixes the order).
    for (uint32_t g = 0; g < ng; ++g) {
      if (group_rows[g] <= 0) continue;
      for (size_t i = 0; i < q.items.size(); ++i) {
        auto& col = res->cols[i];
        const SelItem& it = q.items[i];
        if (it.agg < 0) {
          col.str.push_back(g < dl ? (*key.dict)[g] : std::string());
          col.nulls.push_back(g < dl ? 0 : 1);
        } else {
          const fdb_agg_value& v = vals[i][g];
          if (col.dtype == FDB_INT64) {
            col.i64.push_back(v.i);
            col.nulls.push_back(0);
          } else {
            col.f64.push_back(v.f);
            col.nulls.push_back(v.valid ? 0 : 1);
          }
        }
      }
      ++res->rows;
    }
  } else if (key.dtype == FDB_INT64) {
    // One value column for every aggregate (fast_i64_gb's common shape).
    int vc = -1;
    for (size_t i : agg_items) {
      const SelItem& it = q.items[i];
      if (it.agg == FDB_AGG_COUNT_STAR) continue;
      if (it.agg == FDB_AGG_COUNT) fail(FDB_E_SQL, "use COUNT(*) with an INT64 GROUP BY key");
      const int rc = resolve(rel, it.col);
      if (vc >= 0 && rc != vc) fail(FDB_E_SQL, "INT64 GROUP BY supports aggregates over one value column");
      vc = rc;
    }
    if (vc < 0) vc = kc;
    if (rel.cols[vc].dtype == FDB_UTF8) fail(FDB_E_TYPE, "aggregate over a text column");
    std::vector<fdb_dev_column> pcols = local_cols(rel, local);
    if (pcols.size() > 2) fail(FDB_E_SQL, "GROUP BY with a WHERE over more than 2 columns");
    const uint64_t cap = rel.nrows + 1;
    fdb_group_i64* d = plan.dev<fdb_group_i64>(cap);
    uint64_t* dn = plan.dev<uint64_t>(1);
    std::vector<fdb_group_i64> groups;
    if (rel.nrows > 0) {
      const GbSizing sz = group_by_i64_sizing(plan.c, key.dev, rel.nrows, 0);
      plan.c.ensure_scratch(group_by_i64_scratch(sz, 0.5) + (16u << 20));
      op_group_by_i64(plan.c, key.dev, rel.cols[vc].dev, rel.nrows, prog.data(), (int)prog.size(), pcols.data(),
                      (int)pcols.size(), sz, 0.5, d, cap, dn);
      plan.check();
      groups = plan.to_host(d, plan.one(dn));
    }
    for (const fdb_group_i64& g : groups) {
      if (g.count <= 0) continue;
      for (size_t i = 0; i < q.items.size(); ++i) {
        auto& col = res->cols[i];
        const SelItem& it = q.items[i];
        const bool null_key = g.key == INT64_MIN;
        switch (it.agg) {
          case -1:
            col.i64.push_back(null_key ? 0 : g.key);
            col.nulls.push_back(null_key ? 1 : 0);
            break;
          case FDB_AGG_COUNT_STAR:
            col.i64.push_back(g.count);
            col.nulls.push_back(0);
            break;
          case FDB_AGG_SUM:
            col.f64.push_back(g.sum);
            col.nulls.push_back(0);
            break;
          case FDB_AGG_AVG:
            col.f64.push_back(g.sum / (double)g.count);
            col.nulls.push_back(0);
            break;
          case FDB_AGG_MIN:
            col.f64.push_back(g.min);
            col.nulls.push_back(std::isnan(g.min) ? 1 : 0);
            break;
          case FDB_AGG_MAX:
            col.f64.push_back(g.max);
            col.nulls.push_back(std::isnan(g.max) ? 1 : 0);
            break;
          default: fail(FDB_E_SQL, "aggregate not supported with an INT64 GROUP BY key");
        }
      }
      ++res->rows;
    }
  } else {
    fail(FDB_E_SQL, "GROUP BY over a FLOAT64 column is not supported");
  }
  apply_order_limit(res, order_keys(res, q, q.items), q.limit);
}

// ---------------------------------------------------------------------------
// Projection (SELECT cols [WHERE] [ORDER BY] [LIMIT])
// ---------------------------------------------------------------------------
// The result rows `d_list` (n entries, in output order; null = rows 0..n-1)
// fetched into the result columns; with SELECT DISTINCT (one column) only each
// value's first occurrence in that order is kept (dedup_batches,
// select.rs:238-457).
static void emit_rows(Plan& plan, const Rel& rel, const std::vector<int>& outcols, const Query& q,
                      const uint32_t* d_list, uint64_t n, fdb_result* res) {
  if (q.distinct && n > 0 && outcols.size() > 1) {
    // Whole rows (dedup_batches, select.rs:238-269): the first occurrence of
    // each distinct row of the projected columns, in list order.
    if (outcols.size() > 8) fail(FDB_E_SQL, "SELECT DISTINCT over more than 8 columns is not supported");
    std::vector<fdb_dev_column> cols;
    std::vector<const uint32_t*> ranks;
    std::vector<uint32_t> rank_lens;
    for (int oc : outcols) {
      const RelCol& col = rel.cols[oc];
      cols.push_back(col.dev);
      const bool text = col.dtype == FDB_UTF8 && col.dict;
      ranks.push_back(text ? dict_ranks(plan, col) : nullptr);
      rank_lens.push_back(text ? (uint32_t)col.dict->size() : 0u);
    }
    uint32_t* pos = plan.dev<uint32_t>(n);
    uint64_t* dcount = plan.dev<uint64_t>(1);
    plan.c.scratch_reset();
    op_distinct_multi(plan.c, cols.data(), ranks.data(), rank_lens.data(), (int)cols.size(), d_list, n, pos, dcount);
    plan.c.scratch_reset();
    plan.check();
    const uint64_t k = plan.one(dcount);
    uint32_t* kept = pos;
    if (d_list) {
      kept = plan.dev<uint32_t>(std::max<uint64_t>(k, 1));
      fdb_dev_column list{};
      list.dtype = FDB_UTF8;  // 4-byte gather of row numbers
      list.values = d_list;
      op_gather(plan.c, list, pos, k, kept, nullptr);
    }
    for (size_t i = 0; i < outcols.size(); ++i) fetch_rows(plan, rel, outcols[i], kept, k, res->cols[i]);
    res->rows = k;
    return;
  }
  if (q.distinct && n > 0) {
    const RelCol& col = rel.cols[outcols[0]];
    fdb_dev_column g = col.dev;
    if (d_list) {
      void* vals = plan.dev<uint8_t>(n * dtype_size(col.dtype));
      uint64_t* valid = col.dev.validity ? plan.dev<uint64_t>((n + 63) / 64) : nullptr;
      op_gather(plan.c, col.dev, d_list, n, vals, valid);
      g = fdb_dev_column{};
      g.dtype = col.dtype;
      g.values = vals;
      g.validity = valid;
    }
    uint32_t* pos = plan.dev<uint32_t>(n);
    uint64_t* dcount = plan.dev<uint64_t>(1);
    op_distinct(plan.c, g, n, pos, dcount);
    plan.c.scratch_reset();  // the sort's working memory is free for the next operator
    plan.check();
    const uint64_t k = plan.one(dcount);
    uint32_t* kept = pos;
    if (d_list) {
      kept = plan.dev<uint32_t>(std::max<uint64_t>(k, 1));
      fdb_dev_column list{};
      list.dtype = FDB_UTF8;  // 4-byte gather of row numbers
      list.values = d_list;
      op_gather(plan.c, list, pos, k, kept, nullptr);
    }
    fetch_rows(plan, rel, outcols[0], kept, k, res->cols[0]);
    res->rows = k;
    if (col.dtype == FDB_UTF8) {
      // Codes name strings; a dictionary that holds one string under two codes
      // still yields the string once (value semantics, row_eq on get_str).
      fdb_result::Col& rc = res->cols[0];
      std::set<std::string> seen;
      bool null_seen = false;
      fdb_result::Col out;
      out.name = rc.name;
      out.dtype = rc.dtype;
      for (uint64_t i = 0; i < k; ++i) {
        const bool is_null = !rc.nulls.empty() && rc.nulls[i];
        if (is_null ? std::exchange(null_seen, true) : !seen.insert(rc.str[i]).second) continue;
        out.str.push_back(rc.str[i]);
        out.nulls.push_back(is_null ? 1 : 0);
      }
      res->rows = out.str.size();
      rc = std::move(out);
    }
    return;
  }
  for (size_t i = 0; i < outcols.size(); ++i) fetch_rows(plan, rel, outcols[i], d_list, n, res->cols[i]);
  res->rows = n;
}

static void run_projection(Plan& plan, const Rel& rel_in, const Query& q, fdb_result* res) {
  // The relation plus one INT64 column per ROW_NUMBER() item, filled once the
  // WHERE survivors are known (windows run after WHERE, db.rs:1660-1697).
  Rel rel;
  rel.nrows = rel_in.nrows;
  rel.cols = rel_in.cols;
  std::vector<std::pair<int, const SelItem*>> windows;  // (rel column, item)
  // Output column list.
  std::vector<int> outcols;
  std::vector<SelItem> items;
  for (const SelItem& it : q.items) {
    if (it.agg >= 0) fail(FDB_E_SQL, "mixing aggregates and plain columns needs GROUP BY");
    if (it.row_number) {
      RelCol rc;
      rc.name = it.alias.empty() ? std::string("row_number") : it.alias;
      rc.dtype = FDB_INT64;
      rc.dev.dtype = FDB_INT64;
      rc.dev.values = plan.dev<int64_t>(std::max<uint64_t>(rel.nrows, 1));
      rel.cols.push_back(rc);
      windows.push_back({(int)rel.cols.size() - 1, &it});
      outcols.push_back((int)rel.cols.size() - 1);
      items.push_back(it);
      continue;
    }
    if (it.star) {
      for (size_t i = 0; i < rel.cols.size(); ++i) {
        outcols.push_back((int)i);
        SelItem s;
        s.col.col = rel.cols[i].name;
        s.text = rel.cols[i].name;
        items.push_back(s);
      }
    } else {
      outcols.push_back(resolve(rel, it.col));
      items.push_back(it);
    }
  }
  for (size_t i = 0; i < outcols.size(); ++i) push_col(res, out_name(items[i]), rel.cols[outcols[i]].dtype);

  // 1. Selected rows (all rows, or the WHERE survivors in row order).
  const uint64_t n = rel.nrows;
  uint32_t* d_rows = nullptr;
  uint64_t nsel = n;
  bool all_rows = true;
  if (q.where && n > 0) {
    std::vector<int> local;
    PredCompiler pc{plan, rel, local, {}};
    pc.compile(*q.where);
    std::vector<fdb_dev_column> cols = local_cols(rel, local);
    uint64_t* mask = plan.dev<uint64_t>((n + 63) / 64);
    op_filter_mask(plan.c, cols.data(), (int)cols.size(), n, pc.terms.data(), (int)pc.terms.size(), mask);
    d_rows = plan.dev<uint32_t>(n);
    uint64_t* dc = plan.dev<uint64_t>(1);
    op_compact_mask(plan.c, mask, n, d_rows, n, dc);
    plan.check();
    nsel = plan.one(dc);
    all_rows = false;
  }

  // ROW_NUMBER() columns: the selected rows numbered 1..nsel in the window's
  // order -- the single-key typed sort (try_dense_partition_sort,
  // window.rs:308-331: f64_ord_key of the value, an INT64 read as f64, NOT for
  // DESC, ties by position) -- or in row order without ORDER BY.
  for (auto& w : windows) {
    int64_t* rn = static_cast<int64_t*>(const_cast<void*>(rel.cols[w.first].dev.values));
    const uint32_t* list = all_rows ? nullptr : d_rows;
    if (!w.second->has_worder || nsel == 0) {
      op_row_numbers(plan.c, nullptr, list, nsel, rn);
      continue;
    }
    const int oc = resolve(rel_in, w.second->worder.ref);
    const RelCol& ocol = rel.cols[oc];
    if (ocol.dtype == FDB_UTF8) fail(FDB_E_SQL, "ROW_NUMBER() OVER (ORDER BY a text column) is not supported");
    if (ocol.dev.validity) fail(FDB_E_SQL, "ROW_NUMBER() OVER (ORDER BY a nullable column) is not supported");
    fdb_dev_column g = ocol.dev;
    if (!all_rows) {
      uint64_t* vals = plan.dev<uint64_t>(nsel);
      op_gather(plan.c, ocol.dev, d_rows, nsel, vals, nullptr);
      g = fdb_dev_column{};
      g.dtype = ocol.dtype;
      g.values = vals;
    }
    uint32_t* order = plan.dev<uint32_t>(nsel);
    op_sort_keyed(plan.c, g, nsel, w.second->worder.desc, false, true, order);
    plan.c.scratch_reset();
    op_row_numbers(plan.c, order, list, nsel, rn);
  }

  // 2. ORDER BY one column + small LIMIT: bounded top-k on the GPU.
  if (q.order.size() == 1 && q.limit >= 1 && q.limit <= 4096 && nsel > 0) {
    const OrderItem& o = q.order[0];
    int oc = -1;
    for (size_t i = 0; i < items.size(); ++i)
      if (items[i].alias == o.ref.col) oc = outcols[i];
    if (oc < 0 && !(o.ref.col.size() && o.ref.col[0] == '#')) oc = resolve(rel, o.ref);
    if (oc >= 0 && rel.cols[oc].dtype != FDB_UTF8) {
      const uint32_t k = (uint32_t)std::min<uint64_t>((uint64_t)q.limit, nsel);
      uint32_t* top = plan.dev<uint32_t>(k);
      uint64_t* dcount = plan.dev<uint64_t>(1);
      if (all_rows) {
        op_topk(plan.c, rel.cols[oc].dev, n, k, o.desc, o.nulls_last, top, dcount);
      } else {
        // Gather the ORDER BY column of the survivors, rank it, map back.
        const RelCol& ocol = rel.cols[oc];
        uint64_t* vals = plan.dev<uint64_t>(nsel);
        uint64_t* valid = ocol.dev.validity ? plan.dev<uint64_t>((nsel + 63) / 64) : nullptr;
        op_gather(plan.c, ocol.dev, d_rows, nsel, vals, valid);
        fdb_dev_column g{};
        g.dtype = ocol.dtype;
        g.values = vals;
        g.validity = valid;
        uint32_t* local_top = plan.dev<uint32_t>(k);
        op_topk(plan.c, g, nsel, k, o.desc, o.nulls_last, local_top, dcount);
        fdb_dev_column rows_col{};
        rows_col.dtype = FDB_UTF8;  // 4-byte gather of row numbers
        rows_col.values = d_rows;
        op_gather(plan.c, rows_col, local_top, k, top, nullptr);
      }
      plan.check();
      const uint64_t got = plan.one(dcount);
      emit_rows(plan, rel, outcols, q, top, got, res);
      return;
    }
  }

  // 3. ORDER BY one FLOAT64 / INT64 column with no LIMIT or a larger one: GPU
  //    radix sort of the selected rows (the single-key typed sort,
  //    try_typed_sort, sort.rs:209-350), then the LIMIT.
  if (q.order.size() == 1 && nsel > 0) {
    const OrderItem& o = q.order[0];
    int oc = -1;
    if (!o.ref.col.empty() && o.ref.col[0] == '#') {
      const int pos = std::atoi(o.ref.col.c_str() + 1) - 1;
      if (pos >= 0 && pos < (int)outcols.size()) oc = outcols[pos];
    } else {
      for (size_t i = 0; i < items.size(); ++i)
        if (items[i].alias == o.ref.col) oc = outcols[i];
      if (oc < 0) oc = resolve(rel, o.ref);
    }
    if (oc >= 0 && rel.cols[oc].dtype != FDB_UTF8) {
      uint32_t* order = plan.dev<uint32_t>(nsel);
      if (all_rows) {
        op_sort(plan.c, rel.cols[oc].dev, n, o.desc, o.nulls_last, order);
        plan.c.scratch_reset();
      } else {
        const RelCol& ocol = rel.cols[oc];
        uint64_t* vals = plan.dev<uint64_t>(nsel);
        uint64_t* valid = ocol.dev.validity ? plan.dev<uint64_t>((nsel + 63) / 64) : nullptr;
        op_gather(plan.c, ocol.dev, d_rows, nsel, vals, valid);
        fdb_dev_column g{};
        g.dtype = ocol.dtype;
        g.values = vals;
        g.validity = valid;
        uint32_t* local = plan.dev<uint32_t>(nsel);
        op_sort(plan.c, g, nsel, o.desc, o.nulls_last, local);
        plan.c.scratch_reset();
        fdb_dev_column rows_col{};
        rows_col.dtype = FDB_UTF8;  // 4-byte gather of row numbers
        rows_col.values = d_rows;
        op_gather(plan.c, rows_col, local, nsel, order, nullptr);
      }
      plan.check();
      const uint64_t take = q.limit >= 0 ? std::min<uint64_t>((uint64_t)q.limit, nsel) : nsel;
      emit_rows(plan, rel, outcols, q, order, take, res);
      return;
    }
  }

  // 4. Several ORDER BY keys, a text key, or a key that is not projected:
  //    stable radix sorts of the selected rows on the GPU, last key first
  //    (sort_merged over several SortExprs, sort.rs:118-165; a text column by
  //    the rank of its code in the sorted dictionary, sort.rs:352-382), then
  //    the LIMIT.
  if (!q.order.empty() && nsel > 0) {
    if (q.order.size() > 8) fail(FDB_E_SQL, "ORDER BY over more than 8 keys is not supported");
    std::vector<SortKey> keys;
    for (const OrderItem& o : q.order) {
      int oc = -1;
      if (!o.ref.col.empty() && o.ref.col[0] == '#') {
        const int pos = std::atoi(o.ref.col.c_str() + 1) - 1;
        if (pos < 0 || pos >= (int)outcols.size()) fail(FDB_E_SQL, "bad ORDER BY reference");
        oc = outcols[pos];
      } else {
        for (size_t i = 0; i < items.size() && oc < 0; ++i)
          if (items[i].alias == o.ref.col || (items[i].col.col == o.ref.col &&
                                              (o.ref.table.empty() || resolve(rel, o.ref) == outcols[i])))
            oc = outcols[i];
        if (oc < 0) oc = resolve(rel, o.ref);
      }
      const RelCol& col = rel.cols[oc];
      SortKey k;
      k.col = col.dev;
      k.desc = o.desc;
      k.nulls_last = o.nulls_last;
      if (col.dtype == FDB_UTF8) {
        if (!col.dict) fail(FDB_E_SQL, "ORDER BY a text column without a dictionary");
        k.rank = dict_ranks(plan, col);
        k.rank_len = (uint32_t)col.dict->size();
      }
      keys.push_back(k);
    }
    uint32_t* pos = plan.dev<uint32_t>(nsel);
    plan.c.scratch_reset();
    op_sort_multi(plan.c, keys.data(), (int)keys.size(), all_rows ? nullptr : d_rows, nsel, pos);
    plan.c.scratch_reset();
    uint32_t* order = pos;
    if (!all_rows) {
      order = plan.dev<uint32_t>(nsel);
      fdb_dev_column rows_col{};
      rows_col.dtype = FDB_UTF8;  // 4-byte gather of row numbers
      rows_col.values = d_rows;
      op_gather(plan.c, rows_col, pos, nsel, order, nullptr);
    }
    plan.check();
    const uint64_t take = q.limit >= 0 ? std::min<uint64_t>((uint64_t)q.limit, nsel) : nsel;
    emit_rows(plan, rel, outcols, q, order, take, res);
    return;
  }

  // 5. No ORDER BY: the selected rows in row order, then the LIMIT.
  uint64_t take = nsel;
  if (q.limit >= 0) take = std::min<uint64_t>(take, (uint64_t)q.limit);
  if (q.distinct) {
    emit_rows(plan, rel, outcols, q, all_rows ? nullptr : d_rows, take, res);
    return;
  }
  if (all_rows) {
    d_rows = plan.dev<uint32_t>(take);
    std::vector<uint32_t> iota(take);
    std::iota(iota.begin(), iota.end(), 0u);
    if (take) FDB_CUDA(cudaMemcpyAsync(d_rows, iota.data(), take * 4, cudaMemcpyHostToDevice, plan.c.stream));
  }
  for (size_t i = 0; i < outcols.size(); ++i) fetch_rows(plan, rel, outcols[i], d_rows, take, res->cols[i]);
  res->rows = take;
}

// ---------------------------------------------------------------------------
// Joins
// ---------------------------------------------------------------------------
struct JoinSpec {
  std::shared_ptr<Table> left, right;   // probe side, build side
  std::string lalias, ralias;
  int type = FDB_JOIN_INNER;
  std::string lkey, rkey;
};

static bool names_side(const ColRef& r, const std::string& table, const std::string& alias) {
  return r.table.empty() || r.table == table || (!alias.empty() && r.table == alias);
}

static void run_join(Plan& plan, Query& q, const JoinSpec& js, fdb_result* res) {
  Ctx& c = plan.c;
  Table& L = *js.left;
  Table& R = *js.right;
  const int lk = L.find(js.lkey), rk = R.find(js.rkey);
  if (lk < 0) fail(FDB_E_NOTFOUND, "no column " + js.lkey + " in " + L.name);
  if (rk < 0) fail(FDB_E_NOTFOUND, "no column " + js.rkey + " in " + R.name);
  const Column& lkc = L.cols[lk];
  const Column& rkc = R.cols[rk];
  if (lkc.dtype != FDB_INT64 || rkc.dtype != FDB_INT64) fail(FDB_E_TYPE, "join keys must both be INT64");
  for (const Column* col : {&lkc, &rkc}) FDB_CUDA(cudaStreamWaitEvent(c.stream, col->ready, 0));

  Rel lrel, rrel;
  add_table_cols(c, lrel, L, js.lalias);
  add_table_cols(c, rrel, R, js.ralias);
  const bool semi_anti = js.type == FDB_JOIN_SEMI || js.type == FDB_JOIN_ANTI;

  // Fast path: COUNT(*) and one SUM, no WHERE (besides the EXISTS itself) and
  // no GROUP BY / ORDER BY.
  bool fast = !q.has_group && q.order.empty() && (!q.where || semi_anti) && !q.items.empty();
  int sum_col = -1;
  const Rel* sum_rel = nullptr;
  for (const SelItem& it : q.items) {
    if (it.agg == FDB_AGG_COUNT_STAR) continue;
    if (it.agg != FDB_AGG_SUM || sum_col >= 0) {
      fast = false;
      break;
    }
    if (semi_anti) {
      sum_rel = &lrel;
    } else if (names_side(it.col, R.name, js.ralias) && R.find(it.col.col) >= 0 &&
               !(it.col.table.empty() && L.find(it.col.col) >= 0)) {
      sum_rel = &rrel;
    } else {
      fast = false;
      break;
    }
    sum_col = resolve(*sum_rel, it.col);
    const int32_t dt = sum_rel->cols[sum_col].dtype;
    if ((semi_anti && dt != FDB_FLOAT64) || (!semi_anti && dt != FDB_INT64)) fast = false;
  }
  // The payload is the summed build column (or none).
  fdb_dev_column payload{};
  if (fast && !semi_anti && sum_col >= 0) payload = rrel.cols[sum_col].dev;
  fdb_dev_column rkey = rrel.cols[rk].dev;
  c.ensure_scratch(64u << 20);
  HashTable* ht = op_join_build(c, rkey, payload, R.nrows, 0.5);
  struct Guard {
    HashTable* h;
    ~Guard() { join_free(h); }
  } guard{ht};
  const fdb_dev_column lkey = lrel.cols[lk].dev;

  if (fast) {
    fdb_join_agg* d = plan.dev<fdb_join_agg>(1);
    const fdb_dev_column* val = (semi_anti && sum_col >= 0) ? &lrel.cols[sum_col].dev : nullptr;
    c.scratch_reset();
    op_join_probe_agg(c, *ht, lkey, val, L.nrows, js.type, d);
    plan.check();
    const fdb_join_agg h = plan.one(d);
    for (const SelItem& it : q.items) {
      if (it.agg == FDB_AGG_COUNT_STAR) {
        push_col(res, out_name(it), FDB_INT64);
        res->cols.back().i64.push_back(h.count);
        res->cols.back().nulls.push_back(0);
      } else {
        push_col(res, out_name(it), FDB_FLOAT64);
        const double s = semi_anti ? h.sum_value : (double)h.sum_payload;
        res->cols.back().f64.push_back(s);
        res->cols.back().nulls.push_back(h.payload_rows > 0 ? 0 : 1);
      }
    }
    res->rows = 1;
    return;
  }

  // General path: emit the row pairs, materialise the joined relation, and run
  // the single-table plan over it.
  c.scratch_reset();
  fdb_join_agg* dcnt = plan.dev<fdb_join_agg>(1);
  op_join_probe_agg(c, *ht, lkey, nullptr, L.nrows,
                    semi_anti ? js.type : (js.type == FDB_JOIN_LEFT ? FDB_JOIN_LEFT : FDB_JOIN_INNER), dcnt);
  plan.check();
  const uint64_t npairs = (uint64_t)plan.one(dcnt).count;
  uint32_t* dl = plan.dev<uint32_t>(npairs);
  uint32_t* dr = semi_anti ? nullptr : plan.dev<uint32_t>(npairs);
  uint64_t* dn = plan.dev<uint64_t>(1);
  c.scratch_reset();
  op_join_probe_pairs(c, *ht, lkey, L.nrows, js.type, dl, dr, npairs, dn);
  plan.check();
  const uint64_t got = plan.one(dn);
  if (got != npairs) fail(FDB_E_GENERIC, "join pair count changed between passes");
  // Pair order from the device is unspecified: order by (left row, right row)
  // so the joined relation is deterministic (the reference probes left rows in
  // order, join.rs:297-375).  The GPU radix sort does it in place.
  c.scratch_reset();
  op_sort_row_pairs(c, dl, dr, npairs);
  c.scratch_reset();

  Rel joined;
  joined.nrows = npairs;
  auto add_side = [&](const Rel& side, const uint32_t* rows, bool optional) {
    for (const RelCol& col : side.cols) {
      RelCol nc = col;
      const int esz = dtype_size(col.dtype);
      void* vals = plan.dev<uint8_t>(npairs * esz);
      uint64_t* valid = nullptr;
      if (optional) {
        valid = plan.dev<uint64_t>((npairs + 63) / 64);
        op_gather_opt(c, col.dev, rows, npairs, vals, valid);
      } else {
        if (col.dev.validity) valid = plan.dev<uint64_t>((npairs + 63) / 64);
        op_gather(c, col.dev, rows, npairs, vals, valid);
      }
      nc.dev.values = vals;
      nc.dev.validity = valid;
      nc.dev.validity_offset = 0;
      joined.cols.push_back(nc);
    }
  };
  add_side(lrel, dl, false);
  if (!semi_anti) add_side(rrel, dr, js.type == FDB_JOIN_LEFT);

  Query rest;
  rest.items = q.items;
  rest.has_group = q.has_group;
  rest.group = q.group;
  rest.order = q.order;
  rest.limit = q.limit;
  rest.distinct = q.distinct;
  // A WHERE beside the JOIN filters the joined rows (the EXISTS form was the
  // join itself).
  if (q.where && !(q.where->kind == P_EXISTS || q.where->kind == P_NOTEXISTS)) rest.where = std::move(q.where);
  bool all_agg = !rest.items.empty();
  for (const SelItem& it : rest.items) all_agg = all_agg && it.agg >= 0;
  if (rest.distinct && (rest.has_group || all_agg))
    fail(FDB_E_SQL, "SELECT DISTINCT with aggregates or GROUP BY is not supported");
  for (const SelItem& it : rest.items)
    if (it.row_number && rest.has_group) fail(FDB_E_SQL, "ROW_NUMBER() with GROUP BY is not supported");
  if (rest.has_group) run_group_by(plan, joined, rest, res);
  else if (all_agg) run_aggregates(plan, joined, rest, res);
  else run_projection(plan, joined, rest, res);
}

// ---------------------------------------------------------------------------
// Entry
// ---------------------------------------------------------------------------
static std::string fmt_f64(double v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
  if (v == std::floor(v) && std::fabs(v) < 1e15) {
    char b[64];
    std::snprintf(b, sizeof b, "%.0f", v);
    return b;
  }
  char b[64];
  for (int prec = 15; prec <= 17; ++prec) {
    std::snprintf(b, sizeof b, "%.*g", prec, v);
    if (std::strtod(b, nullptr) == v) break;
  }
  return b;
}

}  // namespace fdb

void fdb_result::finalize() {
  for (auto& c : cols) {
    if (c.nulls.size() < rows) c.nulls.resize(rows, 0);
    if (c.dtype == FDB_UTF8) {
      c.str_ptrs.clear();
      for (size_t i = 0; i < c.str.size(); ++i) c.str_ptrs.push_back(c.nulls[i] ? nullptr : c.str[i].c_str());
    }
  }
}

const std::string& fdb_result::display_text() {
  if (display_built_) return display_;
  display_built_ = true;
  std::ostringstream o;
  std::vector<std::vector<std::string>> cells(rows, std::vector<std::string>(cols.size()));
  std::vector<size_t> w(cols.size());
  for (size_t j = 0; j < cols.size(); ++j) {
    w[j] = cols[j].name.size();
    for (uint64_t i = 0; i < rows; ++i) {
      std::string s;
      if (cols[j].nulls[i]) s = "NULL";
      else if (cols[j].dtype == FDB_INT64) s = std::to_string(cols[j].i64[i]);
      else if (cols[j].dtype == FDB_FLOAT64) s = fdb::fmt_f64(cols[j].f64[i]);
      else s = cols[j].str[i];
      w[j] = std::max(w[j], s.size());
      cells[i][j] = s;
    }
  }
  auto line = [&] {
    for (size_t j = 0; j < cols.size(); ++j) o << '+' << std::string(w[j] + 2, '-');
    o << "+\n";
  };
  line();
  for (size_t j = 0; j < cols.size(); ++j) o << "| " << cols[j].name << std::string(w[j] - cols[j].name.size() + 1, ' ');
  o << "|\n";
  line();
  for (uint64_t i = 0; i < rows; ++i) {
    for (size_t j = 0; j < cols.size(); ++j) o << "| " << cells[i][j] << std::string(w[j] - cells[i][j].size() + 1, ' ');
    o << "|\n";
  }
  line();
  o << rows << " row" << (rows == 1 ? "" : "s") << "\n";
  display_ = o.str();
  return display_;
}

namespace fdb {

// Zone-map pruning (execute_select's can_skip, select.rs:115-137): the
// relation is narrowed to the batches from the first to the last one that
// the zone maps cannot rule out for the WHERE clause.  Batches ruled out in
// between are still scanned (their rows fail the filter); none that could
// hold a passing row is ever left out, so no result changes.
static void prune_rel(Plan& plan, Rel& rel, const Query& q) {
  if (!plan.c.zone_maps || !q.where || rel.nrows == 0) return;
  std::vector<int> local;
  PredCompiler pc{plan, rel, local, {}, {}};
  pc.compile(*q.where);
  std::vector<const std::vector<fdb_zone>*> zones;
  std::vector<int32_t> dtypes;
  for (int rc : local) {
    const RelCol& col = rel.cols[(size_t)rc];
    zones.push_back(col.src ? &column_zones(plan.c, *col.src) : nullptr);
    dtypes.push_back(col.dtype);
  }
  const uint64_t nb = zone_batches(rel.nrows);
  const std::vector<uint8_t> out =
      zone_rule_out(zones, dtypes, pc.terms.data(), (int)pc.terms.size(), pc.host_sets, nb);
  uint64_t b0 = 0, b1 = nb;
  while (b0 < nb && out[b0]) ++b0;
  while (b1 > b0 && out[b1 - 1]) --b1;
  if (b0 == 0 && b1 == nb) return;
  const uint64_t r0 = b0 * kZoneRows;
  const uint64_t r1 = std::min<uint64_t>(rel.nrows, b1 * kZoneRows);
  if (r1 <= r0) {
    rel.nrows = 0;
    return;
  }
  for (RelCol& col : rel.cols) {
    col.dev.values = static_cast<const char*>(col.dev.values) + r0 * (uint64_t)dtype_size(col.dtype);
    // r0 is a multiple of 65,536, so the validity view stays word-aligned.
    if (col.dev.validity) col.dev.validity += r0 / 64;
  }
  rel.nrows = r1 - r0;
}

fdb_result* run_sql(Ctx& c, const std::string& sql) {
  Parser ps(sql);
  Query q = ps.query();
  std::unique_ptr<fdb_result> res(new fdb_result());
  c.scratch_reset();
  c.ensure_scratch((size_t)64 << 20);
  Plan plan(c);
  FDB_CUDA(cudaEventRecord(c.ev0, c.stream));

  const bool exists = q.where && (q.where->kind == P_EXISTS || q.where->kind == P_NOTEXISTS);
  if (q.has_join || exists) {
    JoinSpec js;
    js.left = find_table(c, q.table);
    js.lalias = q.alias;
    if (q.has_join) {
      js.right = find_table(c, q.jtable);
      js.ralias = q.jalias;
      js.type = q.join_type;
      // ON a = b: whichever side names the right table is the build key.
      const ColRef* a = &q.on_a;
      const ColRef* b = &q.on_b;
      const bool a_right = !a->table.empty() && (a->table == q.jtable || a->table == q.jalias);
      if (a_right) std::swap(a, b);
      js.lkey = a->col;
      js.rkey = b->col;
    } else {
      // [NOT] EXISTS (SELECT .. FROM u WHERE u.k = t.k)  -> SEMI / ANTI.
      const Pred& e = *q.where;
      js.right = find_table(c, e.sub_table);
      js.ralias = e.sub_alias;
      js.type = e.kind == P_EXISTS ? FDB_JOIN_SEMI : FDB_JOIN_ANTI;
      const ColRef* a = &e.sub_a;
      const ColRef* b = &e.sub_b;
      const bool a_inner = !a->table.empty() && (a->table == e.sub_table || a->table == e.sub_alias);
      if (a_inner) std::swap(a, b);
      js.lkey = a->col;
      js.rkey = b->col;
    }
    run_join(plan, q, js, res.get());
  } else {
    Rel rel;
    add_table_cols(c, rel, *find_table(c, q.table), q.alias);
    prune_rel(plan, rel, q);
    c.last_scan_rows = rel.nrows;
    bool all_agg = !q.items.empty();
    for (const SelItem& it : q.items) all_agg = all_agg && it.agg >= 0;
    if (q.distinct && (q.has_group || all_agg))
      fail(FDB_E_SQL, "SELECT DISTINCT with aggregates or GROUP BY is not supported");
    for (const SelItem& it : q.items)
      if (it.row_number && q.has_group) fail(FDB_E_SQL, "ROW_NUMBER() with GROUP BY is not supported");
    if (q.has_group) run_group_by(plan, rel, q, res.get());
    else if (all_agg) run_aggregates(plan, rel, q, res.get());
    else run_projection(plan, rel, q, res.get());
  }
  FDB_CUDA(cudaEventRecord(c.ev1, c.stream));
  FDB_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0.f;
  FDB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  c.last_kernel_ms = ms;
  res->finalize();
  return res.release();
}

}  // namespace fdb
