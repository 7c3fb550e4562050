// plan.hpp — host compiler from the C ABI's post-order predicate/expression
// node arrays into typed device programs (eval.cuh), with the reference's
// type rules and errors.
#pragma once

#include <string>
#include <vector>

#include "eval.cuh"
#include "runtime.hpp"

namespace prism {

// Kind of a compiled top-level expression (one output column).
enum ExprKind : int32_t {
  EK_F64 = 0,      // numeric program, Float64 output
  EK_DEC = 1,      // exact program, Decimal128(38, scale) output
  EK_COLUMN = 2,   // bare ColumnRef: the input column itself
  EK_LITERAL = 3,  // bare Literal: constant column of the literal's type
  EK_CAST = 4,     // IfThen with a non-f64 numeric target type: program then cast
  EK_STR_SELECT = 5,  // IfThen with Utf8 branches: per-row branch choice + gather
};

struct CompiledExpr {
  int32_t kind = EK_F64;
  int32_t begin = 0, end = 0;   // program nodes (EK_F64 / EK_DEC / EK_CAST)
  int32_t scale = 0;
  int32_t out_type = TY_F64;    // EK_CAST target / EK_LITERAL type
  int32_t column = -1;          // EK_COLUMN
  prism_scalar literal{};       // EK_LITERAL
  std::string literal_str;
  // EK_STR_SELECT: branch sources (column index or literal) + clause ranges
  std::vector<int32_t> branch_cols;       // -1 = literal
  std::vector<std::string> branch_lits;
  int32_t sel_clause_begin = 0, sel_n_clauses = 0;
  bool sel_has_else = false;
};

struct Program {
  std::vector<int> cols;   // program column slot -> batch column index
  std::vector<PNode> pnodes;
  std::vector<PRange> clauses;
  std::vector<ENode> enodes;
  std::vector<std::string> strings;   // per PNode index with bytes (parallel, "" otherwise)
  std::vector<int> string_node;       // pnode index owning strings[i]
  bool has_filter = false;
  PRange filter{0, 0};
  std::vector<CompiledExpr> exprs;

  // device copies (after upload)
  MemP dev;
  const PNode* d_pnodes = nullptr;
  const ENode* d_enodes = nullptr;
  const PRange* d_clauses = nullptr;
  const DCol* d_cols = nullptr;

  int slot_of(int batch_col);
};

// Compiles an optional filter predicate and expressions against `b`'s schema.
Program compile_program(const Batch& b, const prism_predicate* pred, const prism_expr* exprs, int n_exprs,
                        int arith_mode);
// Adds a predicate to an existing program (returns its range in pnodes).
PRange compile_predicate_into(Program& p, const Batch& b, const prism_pred_node* nodes, int n);
// Uploads programs + column views (views of `b`) to the device.
void upload_program(Ctx& ctx, Program& p, const Batch& b);

}  // namespace prism
