/* Jacobian curve formulas for y^2 = x^3 + b (a = 0), instantiated for G1 (Fp)
 * and G2 (Fp2) by oracle_curve.c (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Formulas follow the same Jacobian model as the reference
 * (include/fp_bn254.cuh:871-1022, include/fp2_bn254.cuh:224-403):
 * doubling dbl-2009-l, addition add-2007-bl, mixed addition madd-2007-bl
 * (Explicit-Formulas Database), with P == Q -> double and P == -Q -> infinity.
 *
 * Required macros: PT (struct name), PFX (function prefix), W (limbs per
 * coordinate), FADD/FSUB/FMUL/FZERO(a)/FINV, FONE (pointer to Montgomery 1).
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(PFX, name)

static int FN(is_inf)(const PT* p) { return FZERO(p->z); }

void FN(set_inf)(PT* p) {
  memset(p, 0, sizeof(*p));
  memcpy(p->x, FONE, 8 * W);
  memcpy(p->y, FONE, 8 * W);
}

void FN(dbl)(PT* r, const PT* p) {
  if (FN(is_inf)(p)) { *r = *p; return; }
  uint64_t A[W], B[W], C[W], D[W], E[W], Fv[W], t[W], x3[W], y3[W], z3[W];
  FMUL(A, p->x, p->x);
  FMUL(B, p->y, p->y);
  FMUL(C, B, B);
  FADD(t, p->x, B);
  FMUL(t, t, t);
  FSUB(t, t, A);
  FSUB(t, t, C);
  FADD(D, t, t);
  FADD(E, A, A);
  FADD(E, E, A);
  FMUL(Fv, E, E);
  FSUB(x3, Fv, D);
  FSUB(x3, x3, D);
  FSUB(t, D, x3);
  FMUL(y3, E, t);
  FADD(t, C, C);
  FADD(t, t, t);
  FADD(t, t, t);
  FSUB(y3, y3, t);
  FMUL(z3, p->y, p->z);
  FADD(z3, z3, z3);
  memcpy(r->x, x3, 8 * W);
  memcpy(r->y, y3, 8 * W);
  memcpy(r->z, z3, 8 * W);
}

void FN(add)(PT* r, const PT* p, const PT* q) {
  if (FN(is_inf)(p)) { *r = *q; return; }
  if (FN(is_inf)(q)) { *r = *p; return; }
  uint64_t z1z1[W], z2z2[W], u1[W], u2[W], s1[W], s2[W], h[W], i_[W], j[W], rr[W], v[W], t[W];
  uint64_t x3[W], y3[W], z3[W];
  FMUL(z1z1, p->z, p->z);
  FMUL(z2z2, q->z, q->z);
  FMUL(u1, p->x, z2z2);
  FMUL(u2, q->x, z1z1);
  FMUL(s1, p->y, q->z);
  FMUL(s1, s1, z2z2);
  FMUL(s2, q->y, p->z);
  FMUL(s2, s2, z1z1);
  FSUB(h, u2, u1);
  FSUB(rr, s2, s1);
  if (FZERO(h)) {
    if (FZERO(rr)) { FN(dbl)(r, p); return; }
    FN(set_inf)(r);
    return;
  }
  FADD(i_, h, h);
  FMUL(i_, i_, i_);
  FMUL(j, h, i_);
  FADD(rr, rr, rr);
  FMUL(v, u1, i_);
  FMUL(x3, rr, rr);
  FSUB(x3, x3, j);
  FSUB(x3, x3, v);
  FSUB(x3, x3, v);
  FSUB(t, v, x3);
  FMUL(y3, rr, t);
  FMUL(t, s1, j);
  FADD(t, t, t);
  FSUB(y3, y3, t);
  FADD(z3, p->z, q->z);
  FMUL(z3, z3, z3);
  FSUB(z3, z3, z1z1);
  FSUB(z3, z3, z2z2);
  FMUL(z3, z3, h);
  memcpy(r->x, x3, 8 * W);
  memcpy(r->y, y3, 8 * W);
  memcpy(r->z, z3, 8 * W);
}

void FN(add_aff)(PT* r, const PT* p, const uint64_t* qx, const uint64_t* qy) {
  if (FZERO(qx) && FZERO(qy)) { *r = *p; return; }
  if (FN(is_inf)(p)) {
    memcpy(r->x, qx, 8 * W);
    memcpy(r->y, qy, 8 * W);
    memcpy(r->z, FONE, 8 * W);
    return;
  }
  uint64_t z1z1[W], u2[W], s2[W], h[W], hh[W], i_[W], j[W], rr[W], v[W], t[W];
  uint64_t x3[W], y3[W], z3[W];
  FMUL(z1z1, p->z, p->z);
  FMUL(u2, qx, z1z1);
  FMUL(s2, qy, p->z);
  FMUL(s2, s2, z1z1);
  FSUB(h, u2, p->x);
  FSUB(rr, s2, p->y);
  if (FZERO(h)) {
    if (FZERO(rr)) { FN(dbl)(r, p); return; }
    FN(set_inf)(r);
    return;
  }
  FMUL(hh, h, h);
  FADD(i_, hh, hh);
  FADD(i_, i_, i_);
  FMUL(j, h, i_);
  FADD(rr, rr, rr);
  FMUL(v, p->x, i_);
  FMUL(x3, rr, rr);
  FSUB(x3, x3, j);
  FSUB(x3, x3, v);
  FSUB(x3, x3, v);
  FSUB(t, v, x3);
  FMUL(y3, rr, t);
  FMUL(t, p->y, j);
  FADD(t, t, t);
  FSUB(y3, y3, t);
  FADD(z3, p->z, h);
  FMUL(z3, z3, z3);
  FSUB(z3, z3, z1z1);
  FSUB(z3, z3, hh);
  memcpy(r->x, x3, 8 * W);
  memcpy(r->y, y3, 8 * W);
  memcpy(r->z, z3, 8 * W);
}

/* affine (x, y) out; (0, 0) and return 1 for infinity */
int FN(to_aff)(uint64_t* out, const PT* p) {
  if (FN(is_inf)(p)) { memset(out, 0, 16 * W); return 1; }
  uint64_t zi[W], zi2[W], zi3[W];
  FINV(zi, p->z);
  FMUL(zi2, zi, zi);
  FMUL(zi3, zi2, zi);
  FMUL(out, p->x, zi2);
  FMUL(out + W, p->y, zi3);
  return 0;
}

#undef FN
#undef CAT
#undef CAT_
