// linalg.cuh -- spinor linear algebra entry points shared with the inverters.
#pragma once

namespace hrgpu {

enum {
  LA_MUL_ADD_ASSIGN = 0, LA_MULC_ADD_ASSIGN, LA_G5_MULC_ADD_ASSIGN, LA_MUL, LA_MULC, LA_ADD, LA_SUB,
  LA_ADD_ASSIGN, LA_SUB_ASSIGN, LA_COPY, LA_ZERO, LA_MINUS, LA_LC, LA_LC_ADD_ASSIGN, LA_CLC,
  LA_CLC_ADD_ASSIGN, LA_G5, LA_G5_ASSIGN, LA_G0, LA_G1, LA_G2, LA_G3, LA_LC1, LA_LC2, LA_LC3
};

int la_check(int par, int prec);
// s1 <- op(s1, s2, s3; c1, c2)
int la_op(int op, int par, int prec, void *s1, const void *s2, const void *s3, double c1r, double c1i, double c2r,
          double c2i);
// op 0: <s1,s2> -> res[0..1] (re, im); 1: <g5 s1, s2> -> res[0..1]; 2: |s1|^2 -> res[0] only
int la_dot(int op, int par, int prec, const void *s1, const void *s2, double *res);

}  // namespace hrgpu
