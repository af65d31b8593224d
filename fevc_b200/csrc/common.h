// Shared host definitions: error codes crossing the C ABI, typed errors and
// the two compensated-summation disciplines the estimator uses.
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace fevcb {

// Stable error classes crossing the C boundary.  The numeric values are the
// reference's `ErrorCode` (rust/crates/vckss-core/src/error.rs:8-48) so that a
// caller written against the reference plugin interprets every status the same.
enum Code : int32_t {
  OK = 0,
  USER_BREAK = 1,
  ABI_MISMATCH = 10,
  UNSUPPORTED_FEATURE = 11,
  INVALID_INPUT = 20,
  INVALID_IDENTIFIER = 21,
  INVALID_WEIGHT = 22,
  INVALID_TARGET_WEIGHT = 23,
  GRAPH_EMPTY = 30,
  GRAPH_UNIDENTIFIED = 31,
  GRAPH_CERTIFICATE_FAILED = 32,
  RESOURCE_LIMIT = 40,
  ALLOCATION_FAILED = 41,
  CMG_SETUP_FAILED = 50,
  CMG_APPLY_FAILED = 51,
  PCG_CURVATURE_BREAKDOWN = 60,
  PCG_PRECONDITIONER_BREAKDOWN = 61,
  PCG_STAGNATION = 62,
  PCG_MAX_ITERATIONS = 63,
  FULL_RESIDUAL_FAILED = 64,
  RNG_CONTRACT_FAILED = 70,
  CORRECTION_NONFINITE = 71,
  ACCOUNTING_IDENTITY_FAILED = 72,
  JLA_MOMENT_FAILED = 73,
  JLA_CONSTRAINT_FAILED = 74,
  NONESTIMABLE_DELETION = 75,
  BLOCK_INVERSE_FAILED = 76,
  TARGET_CENTERING_FAILED = 77,
  TARGET_IDENTITY_FAILED = 78,
  NONFINITE_CORRECTED_TARGET = 79,
  STALE_CONTEXT = 80,
  CONTEXT_POISONED = 81,
  SINGULAR_INFORMATION = 82,
  INVERSE_RESIDUAL_FAILED = 83,
  SYMMETRIC_EIGENSOLVER_FAILED = 86,
  INTERNAL_INVARIANT_FAILED = 90,
  PANIC = 99,
};

// Status-code names as the plugin prints them (reference
// vckss-core/src/error.rs:52-95).
inline const char* code_name(int32_t c) {
  switch (c) {
    case OK: return "OK";
    case USER_BREAK: return "USER_BREAK";
    case ABI_MISMATCH: return "ABI_MISMATCH";
    case UNSUPPORTED_FEATURE: return "UNSUPPORTED_FEATURE";
    case INVALID_INPUT: return "INVALID_INPUT";
    case INVALID_IDENTIFIER: return "INVALID_IDENTIFIER";
    case INVALID_WEIGHT: return "INVALID_WEIGHT";
    case INVALID_TARGET_WEIGHT: return "INVALID_TARGET_WEIGHT";
    case GRAPH_EMPTY: return "GRAPH_EMPTY";
    case GRAPH_UNIDENTIFIED: return "GRAPH_UNIDENTIFIED";
    case GRAPH_CERTIFICATE_FAILED: return "GRAPH_CERTIFICATE_FAILED";
    case RESOURCE_LIMIT: return "RESOURCE_LIMIT";
    case ALLOCATION_FAILED: return "ALLOCATION_FAILED";
    case CMG_SETUP_FAILED: return "CMG_SETUP_FAILED";
    case CMG_APPLY_FAILED: return "CMG_APPLY_FAILED";
    case PCG_CURVATURE_BREAKDOWN: return "PCG_BREAKDOWN_CURVATURE";
    case PCG_PRECONDITIONER_BREAKDOWN: return "PCG_BREAKDOWN_PRECONDITIONER";
    case PCG_STAGNATION: return "PCG_STAGNATION";
    case PCG_MAX_ITERATIONS: return "PCG_MAXITER";
    case FULL_RESIDUAL_FAILED: return "FULL_RESIDUAL_FAILED";
    case RNG_CONTRACT_FAILED: return "RNG_CONTRACT_FAILED";
    case CORRECTION_NONFINITE: return "CORRECTION_NONFINITE";
    case ACCOUNTING_IDENTITY_FAILED: return "ACCOUNTING_IDENTITY_FAILED";
    case JLA_MOMENT_FAILED: return "JLA_MOMENT_FAILED";
    case JLA_CONSTRAINT_FAILED: return "JLA_CONSTRAINT_FAILED";
    case NONESTIMABLE_DELETION: return "NONESTIMABLE_DELETION";
    case BLOCK_INVERSE_FAILED: return "BLOCK_INVERSE_FAILED";
    case TARGET_CENTERING_FAILED: return "TARGET_CENTERING_FAILED";
    case TARGET_IDENTITY_FAILED: return "TARGET_IDENTITY_FAILED";
    case NONFINITE_CORRECTED_TARGET: return "NONFINITE_CORRECTED_TARGET";
    case STALE_CONTEXT: return "STALE_CONTEXT";
    case CONTEXT_POISONED: return "CONTEXT_POISONED";
    case SINGULAR_INFORMATION: return "SINGULAR_INFORMATION";
    case INVERSE_RESIDUAL_FAILED: return "INVERSE_RESIDUAL_FAILED";
    case SYMMETRIC_EIGENSOLVER_FAILED: return "SYMMETRIC_EIGENSOLVER_FAILED";
    case INTERNAL_INVARIANT_FAILED: return "INTERNAL_INVARIANT_FAILED";
    case PANIC: return "PANIC";
    default: return "UNKNOWN";
  }
}

// An error carries its status code; its text reads "NAME [phase]: message"
// like the plugin's last-error string (reference error.rs:125-135).
struct Error : std::runtime_error {
  int32_t code;
  Error(int32_t c, const std::string& phase, const std::string& msg)
      : std::runtime_error(std::string(code_name(c)) + " [" + phase + "]: " + msg), code(c) {}
};

[[noreturn]] inline void fail(int32_t code, const char* phase, const std::string& msg) {
  throw Error(code, phase, msg);
}

constexpr uint64_t MAX_EXACT_BINARY64_INTEGER = uint64_t(1) << 53;

// Neumaier-compensated sum (reference `StableSum`, vckss-core/src/jla.rs:890-905
// and engine.rs:331-352).  Used for every per-unit / per-stratum aggregate.
struct StableSum {
  double sum = 0.0, corr = 0.0;
  void add(double v) {
    double t = sum + v;
    corr += (std::fabs(sum) >= std::fabs(v)) ? (sum - t) + v : (v - t) + sum;
    sum = t;
  }
  double finish() const { return sum + corr; }
};

// Kahan-compensated sum (reference `compensated_sum_interrupt`,
// vckss-core/src/problem.rs:1254-1270).  Used for the compression cell moments.
struct KahanSum {
  double sum = 0.0, corr = 0.0;
  void add(double v) {
    double adj = v - corr;
    double next = sum + adj;
    corr = (next - sum) - adj;
    sum = next;
  }
  double finish() const { return sum; }
};

// Map -0.0 to +0.0 (reference `canonical_zero`, jla.rs:874-880).
inline double canonical_zero(double v) { return v == 0.0 ? 0.0 : v; }

// IEEE-754 totalOrder comparison of binary64 values (Rust `f64::total_cmp`).
inline int total_cmp(double a, double b) {
  int64_t ia, ib;
  static_assert(sizeof(double) == 8, "binary64");
  __builtin_memcpy(&ia, &a, 8);
  __builtin_memcpy(&ib, &b, 8);
  ia ^= int64_t(uint64_t(ia >> 63) >> 1);
  ib ^= int64_t(uint64_t(ib >> 63) >> 1);
  return ia < ib ? -1 : (ia > ib ? 1 : 0);
}

inline int ordered_f64(double a, double b) { return total_cmp(canonical_zero(a), canonical_zero(b)); }

}  // namespace fevcb
