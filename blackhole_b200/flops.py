"""Algorithmic floating-point work of the trace kernel, counted from its source.

Unit of work: one accepted DP5(4) step of one ray (rejected attempts, ray
set-up and event bisection are overhead).  The counts below are the add, sub
and mul operations of the expressions in blackhole_b200/csrc/bh_kernels.cu
(``rhs``, the stage combinations and the error norm of ``attempt``, and the
invariant diagnostics of an accepted step), each counted once per evaluation
with loop-invariant sub-expressions counted once; a fused multiply-add counts
as 2, the same convention as the FMA peak (2 FLOP per FMA).  Divisions,
reciprocals, square roots, sin/cos and pow are listed separately ("special")
and not included in the FLOP figure.

  rhs (per call):        55 real ops + 6 binary64 ops (Sigma, Delta)
                         + 1 sincos + 3 reciprocals
  per attempt:           6 rhs = 330 real + 36 f64
                         stage combinations: 13 + 30 + 42 + 54 + 66 + 66 = 271 real
                         error estimate: 6 x 12 = 72 real; norm: 6 x 4 + 1 = 25 f64,
                         6 divisions, 1 sqrt, 1 pow
  per accepted step:     diagnostics 43 f64, 2 divisions

"real" is binary32 in the mixed path and binary64 in the FP64 path.
"""

RHS_REAL = 55
RHS_F64 = 6
STAGES_REAL = 13 + 30 + 42 + 54 + 66 + 66
ERROR_REAL = 6 * 12
ERROR_F64 = 6 * 4 + 1
DIAG_F64 = 43

PER_ATTEMPT_REAL = 6 * RHS_REAL + STAGES_REAL + ERROR_REAL          # 673
PER_ATTEMPT_F64 = 6 * RHS_F64 + ERROR_F64                           # 61

# FLOPs per accepted step charged against the ALU peak of the path's main pipe.
FLOPS_PER_STEP = {
    # mixed: binary32 work against the FP32 peak; binary64 islands listed apart
    "mixed": {"alu_flop": PER_ATTEMPT_REAL, "f64_flop": PER_ATTEMPT_F64 + DIAG_F64,
              "special": {"sincos": 6, "rcp": 18, "div_f64": 8, "sqrt_f64": 1, "pow_f32": 1}},
    # fp64: everything binary64 against the FP64 peak
    "fp64": {"alu_flop": PER_ATTEMPT_REAL + PER_ATTEMPT_F64 + DIAG_F64, "f64_flop": 0,
             "special": {"sincos": 6, "div_f64": 26, "sqrt_f64": 1, "pow_f64": 1}},
}
