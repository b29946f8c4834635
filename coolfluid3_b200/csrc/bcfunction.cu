// bcfunction.cu -- Dirichlet values given by a function of the node
// coordinates and time (BCDirichletFunction, plugins/UFEM/src/UFEM/
// BCDirichletFunction.cpp:61-92: nodes_expression(dirichlet(var) = f(x, y, z, t))
// with f a parsed function of ParsedFunctionExpression).
//
// The expression text is compiled once on the host into postfix byte code
// (recursive descent: + - * / ^, unary minus below ^, parentheses, the
// variables x y z t, the constant pi and the functions sin cos tan asin acos
// atan sinh cosh tanh exp log sqrt abs).  Every application of the conditions
// evaluates the code on the device for each constrained dof whose first or
// last application is a function, at the handle's current time, with CUDA's
// double-precision math functions; the results replace those dofs' values
// before the symmetric Dirichlet passes (so a function value enters exactly
// as a constant one would).

#include <cuda_runtime.h>

#include <cctype>
#include <cstdlib>
#include <string>
#include <vector>

#include "internal.h"

namespace ufem {
namespace {

enum Op : int32_t {
  kPushConst = 0, kPushX, kPushY, kPushZ, kPushT, kAdd, kSub, kMul, kDiv, kPow, kNeg,
  kSin, kCos, kTan, kAsin, kAcos, kAtan, kSinh, kCosh, kTanh, kExp, kLog, kSqrt, kAbs
};

struct Compiler {
  const std::string& s;
  size_t i = 0;
  std::vector<int32_t>& code;
  std::vector<double>& consts;
  int depth = 0, max_depth = 0;
  std::string err;

  Compiler(const std::string& src, std::vector<int32_t>& c, std::vector<double>& k) : s(src), code(c), consts(k) {}

  void skip() {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m + " at position " + std::to_string(i) + " of \"" + s + "\"";
    return false;
  }
  void emit(int32_t op, int32_t arg = 0) {
    code.push_back(op | (arg << 8));
    if (op <= kPushT) ++depth;
    else if (op >= kAdd && op <= kPow) --depth;
    if (depth > max_depth) max_depth = depth;
  }
  bool expr() {
    if (!term()) return false;
    for (;;) {
      skip();
      if (i < s.size() && (s[i] == '+' || s[i] == '-')) {
        const char o = s[i++];
        if (!term()) return false;
        emit(o == '+' ? kAdd : kSub);
      } else {
        return true;
      }
    }
  }
  bool term() {
    if (!unary()) return false;
    for (;;) {
      skip();
      if (i < s.size() && (s[i] == '*' || s[i] == '/')) {
        const char o = s[i++];
        if (!unary()) return false;
        emit(o == '*' ? kMul : kDiv);
      } else {
        return true;
      }
    }
  }
  bool unary() {
    skip();
    if (i < s.size() && (s[i] == '-' || s[i] == '+')) {
      const char o = s[i++];
      if (!unary()) return false;
      if (o == '-') emit(kNeg);
      return true;
    }
    return power();
  }
  bool power() {
    if (!primary()) return false;
    skip();
    if (i < s.size() && s[i] == '^') {
      ++i;
      if (!unary()) return false;  // right-associative; the exponent may carry a sign
      emit(kPow);
    }
    return true;
  }
  bool primary() {
    skip();
    if (i >= s.size()) return fail("unexpected end of expression");
    const char c = s[i];
    if (c == '(') {
      ++i;
      if (!expr()) return false;
      skip();
      if (i >= s.size() || s[i] != ')') return fail("expected ')'");
      ++i;
      return true;
    }
    if (std::isdigit(static_cast<unsigned char>(c)) || c == '.') {
      const char* b = s.c_str() + i;
      char* e = nullptr;
      const double v = std::strtod(b, &e);
      if (e == b) return fail("malformed number");
      i += size_t(e - b);
      consts.push_back(v);
      emit(kPushConst, int32_t(consts.size() - 1));
      return true;
    }
    if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
      size_t j = i;
      while (j < s.size() && (std::isalnum(static_cast<unsigned char>(s[j])) || s[j] == '_')) ++j;
      const std::string name = s.substr(i, j - i);
      i = j;
      if (name == "x") { emit(kPushX); return true; }
      if (name == "y") { emit(kPushY); return true; }
      if (name == "z") { emit(kPushZ); return true; }
      if (name == "t") { emit(kPushT); return true; }
      if (name == "pi") {
        consts.push_back(3.14159265358979323846);
        emit(kPushConst, int32_t(consts.size() - 1));
        return true;
      }
      static const struct { const char* n; Op op; } fns[] = {
          {"sin", kSin}, {"cos", kCos}, {"tan", kTan}, {"asin", kAsin}, {"acos", kAcos}, {"atan", kAtan},
          {"sinh", kSinh}, {"cosh", kCosh}, {"tanh", kTanh}, {"exp", kExp}, {"log", kLog}, {"sqrt", kSqrt},
          {"abs", kAbs}};
      for (const auto& f : fns)
        if (name == f.n) {
          skip();
          if (i >= s.size() || s[i] != '(') return fail("expected '(' after " + name);
          ++i;
          if (!expr()) return false;
          skip();
          if (i >= s.size() || s[i] != ')') return fail("expected ')'");
          ++i;
          emit(f.op);
          return true;
        }
      return fail("unknown name '" + name + "'");
    }
    return fail(std::string("unexpected character '") + c + "'");
  }
};

__device__ double eval_code(const int32_t* __restrict__ code, int n, const double* __restrict__ k, double x, double y,
                            double z, double t) {
  double st[kExprMaxDepth];
  int sp = 0;
  for (int i = 0; i < n; ++i) {
    const int32_t w = code[i];
    const int op = w & 255;
    switch (op) {
      case kPushConst: st[sp++] = k[w >> 8]; break;
      case kPushX: st[sp++] = x; break;
      case kPushY: st[sp++] = y; break;
      case kPushZ: st[sp++] = z; break;
      case kPushT: st[sp++] = t; break;
      case kAdd: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
      case kSub: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
      case kMul: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
      case kDiv: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
      case kPow: --sp; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
      case kNeg: st[sp - 1] = -st[sp - 1]; break;
      case kSin: st[sp - 1] = sin(st[sp - 1]); break;
      case kCos: st[sp - 1] = cos(st[sp - 1]); break;
      case kTan: st[sp - 1] = tan(st[sp - 1]); break;
      case kAsin: st[sp - 1] = asin(st[sp - 1]); break;
      case kAcos: st[sp - 1] = acos(st[sp - 1]); break;
      case kAtan: st[sp - 1] = atan(st[sp - 1]); break;
      case kSinh: st[sp - 1] = sinh(st[sp - 1]); break;
      case kCosh: st[sp - 1] = cosh(st[sp - 1]); break;
      case kTanh: st[sp - 1] = tanh(st[sp - 1]); break;
      case kExp: st[sp - 1] = exp(st[sp - 1]); break;
      case kLog: st[sp - 1] = log(st[sp - 1]); break;
      case kSqrt: st[sp - 1] = sqrt(st[sp - 1]); break;
      case kAbs: st[sp - 1] = fabs(st[sp - 1]); break;
      default: break;
    }
  }
  return st[0];
}

// One thread per constrained dof: the values of its first and last application
// when those are functions (fn < 0: a constant, left as planned).
__global__ void dirichlet_function_kernel(int64_t nbc, int neq, const int64_t* __restrict__ bc_dof,
                                          const int32_t* __restrict__ fn_first, const int32_t* __restrict__ fn_last,
                                          const int32_t* __restrict__ code, const int32_t* __restrict__ off,
                                          const double* __restrict__ consts, const double* __restrict__ coords,
                                          double t, double* __restrict__ first, double* __restrict__ last) {
  const int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (u >= nbc) return;
  const int f0 = fn_first[u], f1 = fn_last[u];
  if (f0 < 0 && f1 < 0) return;
  const int64_t node = bc_dof[u] / neq;
  const double x = coords[4 * node], y = coords[4 * node + 1], z = coords[4 * node + 2];
  if (f0 >= 0) first[u] = eval_code(code + off[f0], off[f0 + 1] - off[f0], consts, x, y, z, t);
  if (f1 >= 0) last[u] = eval_code(code + off[f1], off[f1 + 1] - off[f1], consts, x, y, z, t);
}

}  // namespace

int compile_expression(const std::string& src, std::vector<int32_t>& code, std::vector<double>& consts,
                       std::string& err) {
  std::vector<int32_t> c;
  Compiler cp(src, c, consts);
  bool ok = cp.expr();
  cp.skip();
  if (ok && cp.i != src.size()) ok = cp.fail("unexpected trailing text");
  if (ok && cp.max_depth > kExprMaxDepth) ok = cp.fail("expression nests too deeply");
  if (!ok) {
    err = cp.err;
    return UFEM_ERR_ARG;
  }
  code.insert(code.end(), c.begin(), c.end());
  return UFEM_OK;
}

int launch_dirichlet_functions(ufem_ns_handle* h, cudaStream_t s) {
  const DirichletPlan& bp = h->bcp;
  if (!bp.fn_first || bp.nbc == 0) return UFEM_OK;
  dirichlet_function_kernel<<<unsigned((bp.nbc + 127) / 128), 128, 0, s>>>(
      bp.nbc, h->neq, bp.bc_dof, bp.fn_first, bp.fn_last, bp.fn_code, bp.fn_off, bp.fn_const, h->d_coords, h->time,
      bp.bc_first, bp.bc_last);
  UFEM_CUDA_TRY(cudaGetLastError());
  return UFEM_OK;
}

}  // namespace ufem
