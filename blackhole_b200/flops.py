"""Algorithmic floating-point work of the trace kernel, counted from its source.

Unit of work: one accepted DP5(4) step of one ray (rejected attempts, ray
set-up and event location are overhead).  The counts are the add, sub and mul
operations of the expressions in blackhole_b200/csrc/bh_trace.cu, each counted
once per evaluation, loop-invariant sub-expressions once; a fused
multiply-add counts 2, the convention of the FMA peak (2 FLOP per FMA).
Reciprocals, divisions, square roots, sin/cos, pow, log and exp are listed separately
("special") and not counted.

  rhs_sc (per call)        S, D (two-term factors), S*D, S*D*sin^2, iS, iD,
                           1/sin^2 from one reciprocal, K, L', B and the six
                           derivatives: 62 ops + 1 reciprocal
  shift_sincos (stages 2-6) angle addition with Taylor series of sin/cos of the
                           stage increment in Horner form: 20 ops in binary32,
                           34 in binary64
  stage combinations       13 + 30 + 42 + 54 + 66 + 66 = 271 ops
  error estimate           per component 12 (stage combination) + 2 (scale)
                           + 1 (scaled error, times the scale's reciprocal)
                           + 2 (square, sum) = 17, x 6 = 102
  step control             hmax 3, error norm 1, h update 1: 5 ops (binary32 in
                           the mixed kernel, binary64 in the FP64 one)
  diagnostics              the five null-norm terms, their sum and the sum of
                           their magnitudes, Carter's Q against Q0 and the two
                           maximum tests: 37 ops per accepted step (the ray's
                           constants a^2 E^2, L_z^2 and 4 a E L_z once per ray);
                           binary32 in the mixed kernel, binary64 in the FP64 one

The sin/cos of stage 7 (the FSAL stage, the next step's base angle) counts as
one special: a full sincos in binary32, angle addition from the base angle in
binary64 (its 34 ops are not counted, so both paths count the same stages); a
ray's first stage takes a full sincos.
"""

RHS = 62
SHIFT = {"mixed": 20, "fp64": 34}
STAGES = 13 + 30 + 42 + 54 + 66 + 66
ERROR = {"mixed": 6 * 17, "fp64": 6 * 17}
CONTROL = 5
DIAG = 37


def per_step(path: str) -> dict:
    alu = 6 * RHS + 5 * SHIFT[path] + STAGES + ERROR[path]
    if path == "mixed":
        return {"alu_flop": alu + CONTROL + DIAG, "f64_flop": 0,
                "special": {"sincos_f32": 1, "rcp_f32": 6 + 6, "lg2_f32": 1, "ex2_f32": 1}}
    return {"alu_flop": alu + CONTROL + DIAG, "f64_flop": 0,
            "special": {"sincos_f64": 1, "rcp_f64": 6 + 6, "log_f64": 1, "exp_f64": 1}}


# FLOPs per accepted step charged against the ALU peak of each path's main pipe:
# mixed 887 binary32, fp64 957 binary64.
FLOPS_PER_STEP = {"mixed": per_step("mixed"), "fp64": per_step("fp64")}
