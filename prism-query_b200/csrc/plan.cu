// plan.cpp — compiles predicates and scalar expressions into typed device
// programs, applying the reference's type rules:
//   compare_column (native/prism-executor/src/filter_project.rs:346-392)
//   evaluate_scalar_expr (filter_project.rs:216-294) incl. IfThen casting.
#include "plan.hpp"

#include <algorithm>
#include <memory>

namespace prism {

namespace {

bool is_int_like(int t) {
  return t == TY_I8 || t == TY_I16 || t == TY_I32 || t == TY_I64 || t == TY_U8 || t == TY_U16 || t == TY_U32 ||
         t == TY_U64;
}
bool f64_castable(int t) { return is_int_like(t) || t == TY_F32 || t == TY_F64 || t == TY_BOOL || t == TY_DEC128; }

const char* type_name(int t) {
  switch (t) {
    case TY_NULL: return "Null";
    case TY_BOOL: return "Boolean";
    case TY_I8: return "Int8";
    case TY_I16: return "Int16";
    case TY_I32: return "Int32";
    case TY_I64: return "Int64";
    case TY_U8: return "UInt8";
    case TY_U16: return "UInt16";
    case TY_U32: return "UInt32";
    case TY_U64: return "UInt64";
    case TY_F32: return "Float32";
    case TY_F64: return "Float64";
    case TY_DATE32: return "Date32";
    case TY_UTF8: return "Utf8";
    case TY_DEC128: return "Decimal128";
    case TY_DICT: return "Dictionary";
  }
  return "?";
}

int scalar_type(const prism_scalar& s) {
  switch (s.type) {
    case PRISM_SCALAR_INT32: return TY_I32;
    case PRISM_SCALAR_INT64: return TY_I64;
    case PRISM_SCALAR_FLOAT64: return TY_F64;
    case PRISM_SCALAR_UTF8: return TY_UTF8;
    case PRISM_SCALAR_BOOLEAN: return TY_BOOL;
    case PRISM_SCALAR_DATE32: return TY_DATE32;
  }
  fail(PRISM_ERR_INVALID_ARGUMENT, "unknown scalar type");
}

struct ETree {
  const prism_expr_node* nd = nullptr;
  std::vector<std::unique_ptr<ETree>> kids;  // bin: l, r; neg: x; if_then: thens..., else?
};

std::unique_ptr<ETree> parse_expr(const prism_expr& e) {
  std::vector<std::unique_ptr<ETree>> st;
  for (int k = 0; k < e.n_nodes; ++k) {
    auto t = std::make_unique<ETree>();
    t->nd = &e.nodes[k];
    int need = 0;
    switch (t->nd->op) {
      case PRISM_EXPR_COLUMN: case PRISM_EXPR_LITERAL: need = 0; break;
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: case PRISM_EXPR_MUL: case PRISM_EXPR_DIV: need = 2; break;
      case PRISM_EXPR_NEG: need = 1; break;
      case PRISM_EXPR_IF_THEN:
        if (t->nd->n_clauses < 0) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed IfThen");
        need = t->nd->n_clauses + (t->nd->has_else ? 1 : 0);
        break;
      default: fail(PRISM_ERR_INVALID_ARGUMENT, "unknown expression op");
    }
    if ((int)st.size() < need) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
    for (int i = (int)st.size() - need; i < (int)st.size(); ++i) t->kids.push_back(std::move(st[i]));
    st.resize(st.size() - need);
    st.push_back(std::move(t));
  }
  if (st.size() != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
  return std::move(st[0]);
}

struct Compiler {
  Program& p;
  const Batch& b;
  const prism_expr* ex = nullptr;
  int mode = PRISM_ARITH_F64;

  const Column& col(int idx) {
    if (idx < 0 || idx >= (int)b.cols.size())
      fail(PRISM_ERR_INVALID_ARGUMENT, "column index " + std::to_string(idx) + " out of range");
    return *b.cols[idx];
  }

  // ------------------------------------------------------ predicates --
  PRange predicate(const prism_pred_node* nodes, int n) {
    PRange r{(int32_t)p.pnodes.size(), n};
    int depth = 0;
    for (int k = 0; k < n; ++k) {
      const prism_pred_node& nd = nodes[k];
      PNode o{};
      switch (nd.op) {
        case PRISM_PRED_LITERAL:
          o.op = P_LIT;
          o.i = nd.value.i64 ? 1 : 0;
          ++depth;
          break;
        case PRISM_PRED_EQ: case PRISM_PRED_NE: case PRISM_PRED_LT: case PRISM_PRED_LE: case PRISM_PRED_GT:
        case PRISM_PRED_GE: {
          const Column& c = col(nd.column);
          int st = nd.value.type;
          o.col = p.slot_of(nd.column);
          o.cmp = nd.op;  // PRISM_PRED_EQ..GE == C_EQ..C_GE
          if ((c.type == TY_I32 && st == PRISM_SCALAR_INT32) || (c.type == TY_I64 && st == PRISM_SCALAR_INT64) ||
              (c.type == TY_DATE32 && (st == PRISM_SCALAR_DATE32 || st == PRISM_SCALAR_INT32))) {
            o.op = P_CMP_INT;
            o.i = nd.value.i64;
          } else if (c.type == TY_F64 && st == PRISM_SCALAR_FLOAT64) {
            o.op = P_CMP_F64;
            o.f = nd.value.f64;
          } else if (c.type == TY_UTF8 && st == PRISM_SCALAR_UTF8) {
            o.op = P_CMP_STR;
            add_string(nd.value, o);
          } else {
            fail(PRISM_ERR_INVALID_ARGUMENT, std::string("Cannot compare column type ") + type_name(c.type) +
                                                 " with scalar " + type_name(scalar_type(nd.value)));
          }
          ++depth;
          break;
        }
        case PRISM_PRED_IS_NULL: case PRISM_PRED_IS_NOT_NULL:
          col(nd.column);
          o.op = nd.op == PRISM_PRED_IS_NULL ? P_IS_NULL : P_IS_NOT_NULL;
          o.col = p.slot_of(nd.column);
          ++depth;
          break;
        case PRISM_PRED_LIKE: case PRISM_PRED_ILIKE: {
          const Column& c = col(nd.column);
          if (c.type != TY_UTF8)
            fail(PRISM_ERR_INVALID_ARGUMENT,
                 std::string(nd.op == PRISM_PRED_LIKE ? "LIKE" : "ILIKE") + " requires Utf8 column, got " +
                     type_name(c.type));
          o.op = P_LIKE;
          o.col = p.slot_of(nd.column);
          o.cmp = nd.op == PRISM_PRED_ILIKE ? 1 : 0;
          add_string(nd.value, o);
          ++depth;
          break;
        }
        case PRISM_PRED_AND: case PRISM_PRED_OR:
          if (depth < 2) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
          o.op = nd.op == PRISM_PRED_AND ? P_AND : P_OR;
          --depth;
          break;
        case PRISM_PRED_NOT:
          if (depth < 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
          o.op = P_NOT;
          break;
        default:
          fail(PRISM_ERR_INVALID_ARGUMENT, "unknown predicate op");
      }
      if (depth > 32) fail(PRISM_ERR_INVALID_ARGUMENT, "predicate nesting deeper than 32");
      p.pnodes.push_back(o);
    }
    if (depth != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
    return r;
  }

  void add_string(const prism_scalar& s, PNode& o) {
    if (s.type != PRISM_SCALAR_UTF8) fail(PRISM_ERR_INVALID_ARGUMENT, "string literal expected");
    p.strings.emplace_back(s.str ? s.str : "", (size_t)std::max<int64_t>(0, s.str_len));
    p.string_node.push_back((int)p.pnodes.size());
    o.slen = (int32_t)s.str_len;
  }

  // ----------------------------------------------------- expressions --
  int arrow_type(const ETree& t) {
    switch (t.nd->op) {
      case PRISM_EXPR_COLUMN: return col(t.nd->column).type;
      case PRISM_EXPR_LITERAL: return scalar_type(t.nd->literal);
      case PRISM_EXPR_IF_THEN:
        if (t.nd->n_clauses == 0) {
          if (!t.nd->has_else) fail(PRISM_ERR_INVALID_ARGUMENT, "IfThen expression requires at least one clause or an else branch");
          return arrow_type(*t.kids.back());
        }
        return arrow_type(*t.kids[0]);
      default:
        return (mode == PRISM_ARITH_EXACT && exactable(t)) ? TY_DEC128 : TY_F64;
    }
  }

  bool exactable(const ETree& t) {
    if (mode != PRISM_ARITH_EXACT) return false;
    switch (t.nd->op) {
      case PRISM_EXPR_COLUMN: {
        int ty = col(t.nd->column).type;
        return is_int_like(ty) || ty == TY_BOOL || ty == TY_DEC128;
      }
      case PRISM_EXPR_LITERAL:
        return t.nd->literal.type == PRISM_SCALAR_INT32 || t.nd->literal.type == PRISM_SCALAR_INT64 ||
               t.nd->literal.type == PRISM_SCALAR_BOOLEAN;
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: case PRISM_EXPR_MUL:
        return exactable(*t.kids[0]) && exactable(*t.kids[1]) && scale_of(t) <= 38;
      case PRISM_EXPR_NEG: return exactable(*t.kids[0]);
      default: return false;
    }
  }

  int scale_of(const ETree& t) {
    switch (t.nd->op) {
      case PRISM_EXPR_COLUMN: {
        const Column& c = col(t.nd->column);
        return c.type == TY_DEC128 ? c.scale : 0;
      }
      case PRISM_EXPR_LITERAL: return 0;
      case PRISM_EXPR_MUL: return scale_of(*t.kids[0]) + scale_of(*t.kids[1]);
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: return std::max(scale_of(*t.kids[0]), scale_of(*t.kids[1]));
      case PRISM_EXPR_NEG: return scale_of(*t.kids[0]);
    }
    return 0;
  }

  void emit(int op, int c = 0, double f = 0, int64_t lo = 0, int64_t hi = 0, int a = 0, int bb = 0) {
    ENode n{};
    n.op = op;
    n.col = c;
    n.f = f;
    n.lo = lo;
    n.hi = hi;
    n.a = a;
    n.b = bb;
    p.enodes.push_back(n);
  }

  // pushes the exact (int128) value of an exactable subtree; returns its scale
  int emit_exact(const ETree& t) {
    const prism_expr_node& nd = *t.nd;
    switch (nd.op) {
      case PRISM_EXPR_COLUMN: {
        const Column& c = col(nd.column);
        emit(E_COL_I128, p.slot_of(nd.column));
        return c.type == TY_DEC128 ? c.scale : 0;
      }
      case PRISM_EXPR_LITERAL: {
        int64_t v = nd.literal.type == PRISM_SCALAR_BOOLEAN ? (nd.literal.i64 ? 1 : 0) : nd.literal.i64;
        emit(E_LIT_I128, 0, 0, v, v < 0 ? -1 : 0);
        return 0;
      }
      case PRISM_EXPR_MUL: {
        int a = emit_exact(*t.kids[0]);
        int c = emit_exact(*t.kids[1]);
        emit(E_MUL_I);
        return a + c;
      }
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: {
        int so = scale_of(t);
        int a = emit_exact(*t.kids[0]);
        if (a < so) emit(E_SCALE_I, so - a);
        int c = emit_exact(*t.kids[1]);
        if (c < so) emit(E_SCALE_I, so - c);
        emit(nd.op == PRISM_EXPR_ADD ? E_ADD_I : E_SUB_I);
        return so;
      }
      case PRISM_EXPR_NEG: {
        int a = emit_exact(*t.kids[0]);
        emit(E_NEG_I);
        return a;
      }
    }
    fail(PRISM_ERR_INTERNAL, "not exactable");
  }

  // pushes the f64 value of a subtree (arrow cast-to-Float64 semantics)
  void emit_f64(const ETree& t) {
    const prism_expr_node& nd = *t.nd;
    if (exactable(t) && nd.op != PRISM_EXPR_COLUMN && nd.op != PRISM_EXPR_LITERAL) {
      int s = emit_exact(t);
      emit(E_I2F, s);
      return;
    }
    switch (nd.op) {
      case PRISM_EXPR_COLUMN: {
        const Column& c = col(nd.column);
        if (!f64_castable(c.type))
          fail(PRISM_ERR_ARROW, std::string("Cast error: Casting from ") + type_name(c.type) + " to Float64 not supported");
        emit(E_COL_F64, p.slot_of(nd.column));
        return;
      }
      case PRISM_EXPR_LITERAL: {
        const prism_scalar& s = nd.literal;
        if (s.type == PRISM_SCALAR_FLOAT64) emit(E_LIT_F64, 0, s.f64);
        else if (s.type == PRISM_SCALAR_INT32 || s.type == PRISM_SCALAR_INT64) emit(E_LIT_F64, 0, (double)s.i64);
        else if (s.type == PRISM_SCALAR_BOOLEAN) emit(E_LIT_F64, 0, s.i64 ? 1.0 : 0.0);
        else fail(PRISM_ERR_ARROW, std::string("Cast error: Casting from ") + type_name(scalar_type(s)) + " to Float64 not supported");
        return;
      }
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: case PRISM_EXPR_MUL: case PRISM_EXPR_DIV:
        emit_f64(*t.kids[0]);
        emit_f64(*t.kids[1]);
        emit(nd.op == PRISM_EXPR_ADD ? E_ADD_F : nd.op == PRISM_EXPR_SUB ? E_SUB_F : nd.op == PRISM_EXPR_MUL ? E_MUL_F : E_DIV_F);
        return;
      case PRISM_EXPR_NEG:
        emit_f64(*t.kids[0]);
        emit(E_NEG_F);
        return;
      case PRISM_EXPR_IF_THEN: {
        int target = arrow_type(t);
        if (!f64_castable(target)) fail(PRISM_ERR_ARROW, std::string("Cast error: Casting from ") + type_name(target) + " to Float64 not supported");
        emit_select(t, /*exact=*/false, target);
        return;
      }
    }
    fail(PRISM_ERR_INVALID_ARGUMENT, "unknown expression op");
  }

  // raw_slots: the select is a top-level output column of type `target`, so a
  // branch that is a bare column of that type reaches the output uncast and
  // keeps its null rows' raw slots (filter_project.rs:277-288: only branches
  // of another type are cast)
  void emit_select(const ETree& t, bool exact, int target, bool raw_slots = false) {
    const prism_expr_node& nd = *t.nd;
    if (nd.n_clauses == 0) {
      if (exact) emit_exact(*t.kids.back());
      else emit_f64(*t.kids.back());
      return;
    }
    bool int_target = is_int_like(target) || target == TY_DATE32 || target == TY_BOOL;
    for (auto& k : t.kids) {
      if (exact) {
        emit_branch_int(*k);
      } else {
        emit_branch_f64(*k, int_target);
      }
      if (raw_slots && k->nd->op == PRISM_EXPR_COLUMN && arrow_type(*k) == target) p.enodes.back().a = 1;
    }
    int begin = (int)p.clauses.size();
    for (int ci = 0; ci < nd.n_clauses; ++ci) {
      const prism_expr_clause& cl = ex->clauses[nd.clause_begin + ci];
      if (cl.pred_begin < 0 || cl.pred_begin + cl.pred_len > ex->n_preds)
        fail(PRISM_ERR_INVALID_ARGUMENT, "IfThen clause predicate out of range");
      p.clauses.push_back(predicate(ex->preds + cl.pred_begin, cl.pred_len));
    }
    emit(E_SELECT, nd.n_clauses, 0, 0, 0, nd.has_else ? 1 : 0, begin);
  }

  void emit_branch_f64(const ETree& k, bool int_target) {
    int ty = arrow_type(k);
    if (ty == TY_UTF8 || ty == TY_DICT || ty == TY_DATE32 && !int_target)
      fail(PRISM_ERR_ARROW, std::string("Cast error: unsupported cast of IfThen branch from ") + type_name(ty));
    emit_f64(k);
    if (int_target && (ty == TY_F64 || ty == TY_F32 || ty == TY_DEC128)) {
      emit(E_F2I);
      emit(E_I2F, 0);
    }
  }

  // integer-domain branch of an integer-typed IfThen (pushes int128)
  void emit_branch_int(const ETree& k) {
    int ty = arrow_type(k);
    if (is_int_like(ty) || ty == TY_DATE32 || ty == TY_BOOL) {
      if (k.nd->op == PRISM_EXPR_COLUMN) { emit(E_COL_I128, p.slot_of(k.nd->column)); return; }
      if (k.nd->op == PRISM_EXPR_LITERAL) {
        int64_t v = k.nd->literal.type == PRISM_SCALAR_BOOLEAN ? (k.nd->literal.i64 ? 1 : 0) : k.nd->literal.i64;
        emit(E_LIT_I128, 0, 0, v, v < 0 ? -1 : 0);
        return;
      }
      if (k.nd->op == PRISM_EXPR_IF_THEN) { emit_select(k, true, ty); return; }
    }
    if (ty == TY_UTF8 || ty == TY_DICT) fail(PRISM_ERR_ARROW, "Cast error: unsupported cast of IfThen branch from Utf8");
    emit_f64(k);
    emit(E_F2I);
  }

  CompiledExpr top(const prism_expr& e) {
    ex = &e;
    auto t = parse_expr(e);
    return top_tree(*t);
  }

  CompiledExpr top_tree(const ETree& t) {
    CompiledExpr c;
    const prism_expr_node& nd = *t.nd;
    switch (nd.op) {
      case PRISM_EXPR_COLUMN:
        col(nd.column);
        c.kind = EK_COLUMN;
        c.column = nd.column;
        return c;
      case PRISM_EXPR_LITERAL:
        c.kind = EK_LITERAL;
        c.literal = nd.literal;
        c.out_type = scalar_type(nd.literal);
        if (nd.literal.type == PRISM_SCALAR_UTF8)
          c.literal_str.assign(nd.literal.str ? nd.literal.str : "", (size_t)std::max<int64_t>(0, nd.literal.str_len));
        return c;
      case PRISM_EXPR_IF_THEN: {
        if (nd.n_clauses == 0) {
          if (!nd.has_else) fail(PRISM_ERR_INVALID_ARGUMENT, "IfThen expression requires at least one clause or an else branch");
          return top_tree(*t.kids.back());
        }
        int target = arrow_type(*t.kids[0]);
        if (target == TY_UTF8) return str_select(t);
        if (target == TY_DICT) fail(PRISM_ERR_ARROW, "Cast error: dictionary IfThen branches are not supported");
        c.begin = (int)p.enodes.size();
        if (target == TY_F64 || target == TY_F32 || target == TY_DEC128) {
          emit_select(t, false, target, /*raw_slots=*/true);
          c.kind = EK_F64;
          c.out_type = TY_F64;
          if (target != TY_F64) { c.kind = EK_CAST; c.out_type = target; }
        } else {
          emit_select(t, true, target, /*raw_slots=*/true);
          c.kind = EK_CAST;
          c.out_type = target;
        }
        c.end = (int)p.enodes.size();
        return c;
      }
      default:
        c.begin = (int)p.enodes.size();
        if (exactable(t)) {
          c.scale = emit_exact(t);
          c.kind = EK_DEC;
          c.out_type = TY_DEC128;
        } else {
          emit_f64(t);
          c.kind = EK_F64;
          c.out_type = TY_F64;
        }
        c.end = (int)p.enodes.size();
        return c;
    }
  }

  CompiledExpr str_select(const ETree& t) {
    CompiledExpr c;
    c.kind = EK_STR_SELECT;
    c.out_type = TY_UTF8;
    const prism_expr_node& nd = *t.nd;
    for (auto& k : t.kids) {
      if (k->nd->op == PRISM_EXPR_COLUMN && col(k->nd->column).type == TY_UTF8) {
        c.branch_cols.push_back(k->nd->column);
        c.branch_lits.emplace_back();
      } else if (k->nd->op == PRISM_EXPR_LITERAL && k->nd->literal.type == PRISM_SCALAR_UTF8) {
        c.branch_cols.push_back(-1);
        c.branch_lits.emplace_back(k->nd->literal.str ? k->nd->literal.str : "",
                                   (size_t)std::max<int64_t>(0, k->nd->literal.str_len));
      } else {
        fail(PRISM_ERR_ARROW, "Cast error: Utf8 IfThen branches must be Utf8 columns or literals");
      }
    }
    c.sel_has_else = nd.has_else != 0;
    c.sel_n_clauses = nd.n_clauses;
    c.sel_clause_begin = (int)p.clauses.size();
    for (int ci = 0; ci < nd.n_clauses; ++ci) {
      const prism_expr_clause& cl = ex->clauses[nd.clause_begin + ci];
      if (cl.pred_begin < 0 || cl.pred_begin + cl.pred_len > ex->n_preds)
        fail(PRISM_ERR_INVALID_ARGUMENT, "IfThen clause predicate out of range");
      p.clauses.push_back(predicate(ex->preds + cl.pred_begin, cl.pred_len));
    }
    return c;
  }
};

}  // namespace

int Program::slot_of(int batch_col) {
  for (size_t i = 0; i < cols.size(); ++i)
    if (cols[i] == batch_col) return (int)i;
  cols.push_back(batch_col);
  return (int)cols.size() - 1;
}

Program compile_program(const Batch& b, const prism_predicate* pred, const prism_expr* exprs, int n_exprs,
                        int arith_mode) {
  Program p;
  if (arith_mode != PRISM_ARITH_F64 && arith_mode != PRISM_ARITH_EXACT)
    fail(PRISM_ERR_INVALID_ARGUMENT, "unknown arithmetic mode");
  Compiler c{p, b, nullptr, arith_mode};
  if (pred) {
    if (!pred->nodes || pred->n_nodes <= 0) fail(PRISM_ERR_INVALID_ARGUMENT, "empty predicate");
    p.filter = c.predicate(pred->nodes, pred->n_nodes);
    p.has_filter = true;
  }
  for (int i = 0; i < n_exprs; ++i) {
    if (!exprs[i].nodes || exprs[i].n_nodes <= 0) fail(PRISM_ERR_INVALID_ARGUMENT, "empty expression");
    p.exprs.push_back(c.top(exprs[i]));
  }
  return p;
}

PRange compile_predicate_into(Program& p, const Batch& b, const prism_pred_node* nodes, int n) {
  Compiler c{p, b, nullptr, PRISM_ARITH_F64};
  return c.predicate(nodes, n);
}

void upload_program(Ctx& ctx, Program& p, const Batch& b) {
  size_t np = p.pnodes.size(), ne = p.enodes.size(), nc = p.clauses.size(), ncol = p.cols.size();
  size_t off_p = 0;
  size_t off_e = (off_p + np * sizeof(PNode) + 15) & ~size_t(15);
  size_t off_c = (off_e + ne * sizeof(ENode) + 15) & ~size_t(15);
  size_t off_d = (off_c + nc * sizeof(PRange) + 15) & ~size_t(15);
  size_t off_s = (off_d + ncol * sizeof(DCol) + 15) & ~size_t(15);
  size_t sbytes = 0;
  for (auto& s : p.strings) sbytes += s.size() + 1;
  size_t total = off_s + sbytes + 16;
  std::vector<uint8_t> host(total, 0);
  p.dev = ctx.alloc(total);
  uint8_t* base = static_cast<uint8_t*>(p.dev->ptr);
  // strings: patch device pointers into the nodes
  size_t so = off_s;
  std::vector<PNode> nodes = p.pnodes;
  for (size_t i = 0; i < p.strings.size(); ++i) {
    std::memcpy(host.data() + so, p.strings[i].data(), p.strings[i].size());
    nodes[p.string_node[i]].s = base + so;
    so += p.strings[i].size() + 1;
  }
  if (np) std::memcpy(host.data() + off_p, nodes.data(), np * sizeof(PNode));
  if (ne) std::memcpy(host.data() + off_e, p.enodes.data(), ne * sizeof(ENode));
  if (nc) std::memcpy(host.data() + off_c, p.clauses.data(), nc * sizeof(PRange));
  for (size_t i = 0; i < ncol; ++i) {
    DCol v = b.cols[p.cols[i]]->view();
    std::memcpy(host.data() + off_d + i * sizeof(DCol), &v, sizeof(DCol));
  }
  ctx.h2d_staged(base, host.data(), total);  // (copied out of `host` before this returns)
  p.d_pnodes = reinterpret_cast<const PNode*>(base + off_p);
  p.d_enodes = reinterpret_cast<const ENode*>(base + off_e);
  p.d_clauses = reinterpret_cast<const PRange*>(base + off_c);
  p.d_cols = reinterpret_cast<const DCol*>(base + off_d);
}

}  // namespace prism
