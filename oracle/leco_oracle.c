/*
 * leco_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, single-threaded restatement of the reference's integer codec hot
 * path (yhliu918/Learn-to-Compress, "LeCo").  It exists so that tests/, the
 * smoke check and bench.py's cpu_baseline leg can check and time the CUDA
 * product against the reference's algorithm.  The product never links,
 * imports or calls this file.
 *
 * Pinning: tests/test_oracle.py compares every function here against the
 * unmodified reference headers compiled into oracle/_ref/libleco_ref.so
 * (oracle/Makefile), and tests/golden/ holds fixtures generated by that
 * library (tests/golden/gen_golden.py).
 *
 * Every arithmetic step follows the reference line it cites.  The reference is
 * built with -ffp-contract=off here, so each FP64 operation below is a single
 * IEEE round-to-nearest operation (this file must be compiled with
 * -ffp-contract=off as well).  Where the reference relies on x86-64 behaviour of
 * an out-of-range double->integer conversion (C undefined behaviour), the
 * x86-64 result is computed explicitly (x86_f2i, x86_f2u) so that the oracle
 * does not depend on the compiler.
 *
 * s = sizeof(T) (4 or 8).  Values are passed as void* arrays of T.
 */
#include <stdint.h>
#include <string.h>
#include <stddef.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

/* ---- conversions ------------------------------------------------------- */

/* (int64_t)x as compiled for x86-64 (CVTTSD2SI): truncation toward zero; NaN and
 * |x| >= 2^63 give INT64_MIN.  Used wherever the reference converts a double
 * prediction to int64_t / long long (e.g. piecewise_fix_integer_template.h:40,54;
 * bit_read.h:240,1187). */
int64_t x86_f2i(double x) {
  if (x >= -9223372036854775808.0 && x < 9223372036854775808.0) return (int64_t)x;
  return INT64_MIN;
}

/* (uint64_t)x as gcc compiles it for x86-64 without AVX-512: x < 2^63 (or NaN)
 * -> CVTTSD2SI(x); otherwise CVTTSD2SI(x - 2^63) with bit 63 flipped.  Used where
 * the reference converts a prediction straight to T (piecewise_fix_integer_template.h:334,
 * bit_read.h:530, piecewise_cost_merge_integer_template_double_wo_round.h:620,691). */
uint64_t x86_f2u(double x) {
  const double two63 = 9223372036854775808.0;
  if (!(x >= two63)) return (uint64_t)x86_f2i(x);
  return (uint64_t)x86_f2i(x - two63) ^ 0x8000000000000000ull;
}

/* (T)double for T of s bytes (u32 takes the low half of CVTTSD2SI). */
static uint64_t f2T(double x, int s) { return s == 8 ? x86_f2u(x) : (uint64_t)(uint32_t)x86_f2i(x); }

/* bits_int_T: 64 - clzll(v), 0 for v == 0 (lr.h:116-130). */
unsigned oracle_bits(uint64_t v) { return v ? 64u - (unsigned)__builtin_clzll(v) : 0u; }

static uint64_t ld(const void *p, int s, size_t i) {
  return s == 8 ? ((const uint64_t *)p)[i] : (uint64_t)((const uint32_t *)p)[i];
}
static void st(void *p, int s, size_t i, uint64_t v) {
  if (s == 8) ((uint64_t *)p)[i] = v; else ((uint32_t *)p)[i] = (uint32_t)v;
}
static uint64_t tmask(int s) { return s == 8 ? ~0ull : 0xffffffffull; }
static uint64_t rd64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
static double rdf64(const uint8_t *p) { double v; memcpy(&v, p, 8); return v; }
static float rdf32(const uint8_t *p) { float v; memcpy(&v, p, 4); return v; }
static uint64_t rdT(const uint8_t *p, int s) { uint64_t v = 0; memcpy(&v, p, (size_t)s); return v; }

/* ---- fits ---------------------------------------------------------------- */

/* lr_int_T<T>::caltheta (lr.h:66-85): four sequential FP64 sums, then
 * theta1 = (sumxy*m - sumx*sumy) / (sumxx*m - sumx*sumx),
 * theta0 = (sumy - theta1*sumx) / m. */
void oracle_lr_fit(const void *y, int s, int m, double *theta0, double *theta1) {
  double sumx = 0, sumy = 0, sumxy = 0, sumxx = 0;
  for (int i = 0; i < m; i++) {
    double di = (double)i, yi = (double)ld(y, s, (size_t)i);
    sumx = sumx + di;
    sumy = sumy + yi;
    sumxx = sumxx + di * (double)i;
    sumxy = sumxy + di * yi;
  }
  double ccc = sumxy * m - sumx * sumy;
  double xxx = sumxx * m - sumx * sumx;
  *theta1 = ccc / xxx;
  *theta0 = (sumy - *theta1 * sumx) / (double)m;
}

/* andviane::polynomial_regression<2> (polynomial_regression_internals.hpp:79-184):
 * x^k columns built by repeated multiplication (:80-99), X[k] = sum x^k and
 * Y[k] = sum x^k * y as sequential FP64 sums (:111-137), row swaps when
 * B[i][i] < B[k][i] (:144-149), Gaussian elimination (:154-159), back
 * substitution against zero-initialised coefficients (:165-171). */
void oracle_poly2_fit(const void *y, int s, int N, double a[3]) {
  double X[5] = {0, 0, 0, 0, 0}, Y[3] = {0, 0, 0};
  for (int k = 0; k < 5; k++) {
    for (int j = 0; j < N; j++) {
      double xr = 1.0, xj = (double)j;
      if (k >= 1) xr = xj;
      for (int d = 2; d <= k; d++) xr = xr * xj;
      X[k] += xr;
    }
  }
  for (int k = 0; k < 3; k++) {
    for (int j = 0; j < N; j++) {
      double xr = 1.0, xj = (double)j;
      if (k >= 1) xr = xj;
      for (int d = 2; d <= k; d++) xr = xr * xj;
      Y[k] += xr * (double)ld(y, s, (size_t)j);
    }
  }
  double B[3][4];
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) B[i][j] = X[i + j];
    B[i][3] = Y[i];
  }
  for (int i = 0; i < 3; i++)
    for (int k = i + 1; k < 3; k++)
      if (B[i][i] < B[k][i])
        for (int j = 0; j < 4; j++) { double t = B[i][j]; B[i][j] = B[k][j]; B[k][j] = t; }
  for (int i = 0; i < 2; i++)
    for (int k = i + 1; k < 3; k++) {
      double t = B[k][i] / B[i][i];
      for (int j = 0; j < 4; j++) B[k][j] -= t * B[i][j];
    }
  a[0] = a[1] = a[2] = 0.0;
  for (int i = 2; i >= 0; --i) {
    a[i] = B[i][3];
    for (int j = 0; j < 3; j++)
      if (j != i) a[i] -= B[i][j] * a[j];
    a[i] /= B[i][i];
  }
}

/* Polynomial::operator() (Polynomial.tpp:17-28): s = s + xx*a; xx = xx*x. */
double oracle_poly2_eval(const double a[3], double x) {
  double xx = 1, sum = 0;
  for (int i = 0; i < 3; i++) {
    sum = sum + xx * a[i];
    xx = xx * x;
  }
  return sum;
}

/* ---- bit packing --------------------------------------------------------- */

/* Byte length of a packed body of n fields of l bits, as written by
 * write_delta_int_T (bit_write.h:257-323): end = ceil(l*n/8) data bytes, one
 * more byte, then 8 - end%8 zero bytes. */
size_t oracle_body_bytes_signed(unsigned l, size_t n) {
  uint64_t endbit = (uint64_t)l * n, end = (endbit + 7) / 8;
  return (size_t)(end + 1 + (8 - end % 8));
}
/* Same for write_FOR_int_T (bit_write.h:326-390): pad = (32-l)/8 when l <= 32;
 * for l > 32 the reference's pad expression wraps and x86-64 writes no pad. */
size_t oracle_body_bytes_for(unsigned l, size_t n) {
  uint64_t endbit = (uint64_t)l * n, end = (endbit + 7) / 8;
  return (size_t)(end + 1 + (l <= 32 ? (32 - l) / 8 : 0));
}

/* Writes field k = v[k] (already reduced to l bits) LSB-first at bit k*l. */
static void put_field(uint8_t *body, uint64_t bit, unsigned l, uint64_t v) {
  for (unsigned b = 0; b < l; b++, bit++)
    if ((v >> b) & 1u) body[bit >> 3] |= (uint8_t)(1u << (bit & 7));
}
/* Reads l bits LSB-first at bit position `bit`. */
static uint64_t get_field(const uint8_t *body, uint64_t bit, unsigned l) {
  uint64_t v = 0;
  for (unsigned b = 0; b < l; b++, bit++) v |= (uint64_t)((body[bit >> 3] >> (bit & 7)) & 1u) << b;
  return v;
}
/* Signed-magnitude field: low l-1 bits magnitude, bit l-1 = 1 when the value
 * lies above the prediction (bit_write.h:287-290; bit_read.h:243-245). */
static uint64_t sm_field(uint64_t mag, int pos, unsigned l) {
  uint64_t m = (l >= 65) ? ~0ull : ((1ull << (l - 1)) - 1);
  return (mag & m) | ((uint64_t)(pos ? 1 : 0) << (l - 1));
}

/* ---- LeCo fixed-block linear: Leco_int<T> ------------------------------ */

/* Leco_int<T>::encodeArray8_int (piecewise_fix_integer_template.h:27-140).
 * Returns bytes written.  seq_fit = theta from oracle_lr_fit. */
size_t oracle_leco_encode(const void *data, int s, size_t n, uint8_t *out) {
  double t0, t1;
  oracle_lr_fit(data, s, (int)n, &t0, &t1);
  int64_t maxd = INT64_MIN, mind = INT64_MAX;
  for (size_t i = 0; i < n; i++) { /* :38-45 */
    int64_t d = (int64_t)(ld(data, s, i) - (uint64_t)x86_f2i(t0 + t1 * (double)i));
    if (d > maxd) maxd = d;
    if (d < mind) mind = d;
  }
  t0 += (double)(int64_t)((uint64_t)maxd + (uint64_t)mind) / 2.; /* :46 */
  uint64_t maxr = 0;
  for (size_t i = 0; i < n; i++) { /* :51-72 */
    int64_t pred = x86_f2i(t0 + t1 * (double)i);
    uint64_t y = ld(data, s, i), r;
    int pos = s == 8 ? (y > (uint64_t)pred) : ((int64_t)y > pred);
    r = (pos ? y - (uint64_t)pred : (uint64_t)pred - y) & tmask(s);
    if (r > maxr) maxr = r;
  }
  unsigned l = maxr ? oracle_bits(maxr) + 1 : 0; /* :108-117 */
  if (l > 8u * (unsigned)s) l = 8u * (unsigned)s;
  out[0] = (uint8_t)l;
  if (l == 8u * (unsigned)s) { /* :120-128 raw */
    for (size_t i = 0; i < n; i++) { uint64_t y = ld(data, s, i); memcpy(out + 1 + i * (size_t)s, &y, (size_t)s); }
    return 1 + n * (size_t)s;
  }
  memcpy(out + 1, &t0, 8);
  memcpy(out + 9, &t1, 8);
  if (!l) return 17;
  size_t nb = oracle_body_bytes_signed(l, n);
  uint8_t *body = out + 17;
  memset(body, 0, nb);
  for (size_t i = 0; i < n; i++) {
    int64_t pred = x86_f2i(t0 + t1 * (double)i);
    uint64_t y = ld(data, s, i);
    int pos = s == 8 ? (y > (uint64_t)pred) : ((int64_t)y > pred);
    uint64_t r = (pos ? y - (uint64_t)pred : (uint64_t)pred - y) & tmask(s);
    put_field(body, (uint64_t)i * l, l, sm_field(r, pos, l));
  }
  return 17 + nb;
}

/* Leco_int<T>::decodeArray8 (piecewise_fix_integer_template.h:142-204) with
 * read_all_bit_fix (bit_read.h:222-275).  strict_raw = 0 reproduces the
 * reference's bulk rule (raw when l >= 8s-1, :171); strict_raw = 1 treats a
 * block as raw only when l == 8s, the rule the encoder and the random-access
 * path use (:120, :313).  Returns the number of values written. */
size_t oracle_leco_decode(const uint8_t *in, int s, size_t n, void *out, int strict_raw) {
  unsigned l = in[0];
  if (l == 127) { st(out, s, 0, rdT(in + 1, s)); return 1; }
  if (l == 126) { st(out, s, 0, rdT(in + 1, s)); st(out, s, 1, rdT(in + 1 + s, s)); return 2; }
  unsigned raw_from = strict_raw ? 8u * (unsigned)s : 8u * (unsigned)s - 1;
  if (l >= raw_from) { memcpy(out, in + 1, n * (size_t)s); return n; }
  double t0 = rdf64(in + 1), t1 = rdf64(in + 9);
  const uint8_t *body = in + 17;
  for (size_t k = 0; k < n; k++) {
    int64_t pred = x86_f2i(t0 + (double)k * t1);
    uint64_t v = (uint64_t)pred;
    if (l) {
      uint64_t f = get_field(body, (uint64_t)k * l, l);
      uint64_t mag = f & ((1ull << (l - 1)) - 1);
      v = ((f >> (l - 1)) & 1) ? v + mag : v - mag;
    }
    st(out, s, k, v);
  }
  return n;
}

/* Leco_int<T>::randomdecodeArray8 (piecewise_fix_integer_template.h:305-337)
 * with read_bit_fix_int_wo_round (bit_read.h:1170-1199). */
uint64_t oracle_leco_random(const uint8_t *in, int s, int k) {
  unsigned l = in[0];
  if (l == 8u * (unsigned)s) return rdT(in + 1 + (size_t)k * s, s);
  double t0 = rdf64(in + 1), t1 = rdf64(in + 9);
  if (!l) return f2T(t0 + (double)k * t1, s); /* :334, double -> T directly */
  uint64_t f = get_field(in + 17, (uint64_t)k * l, l);
  uint64_t mag = f & ((1ull << (l - 1)) - 1);
  uint64_t v = (uint64_t)x86_f2i(t0 + (double)k * t1);
  v = ((f >> (l - 1)) & 1) ? v + mag : v - mag;
  return v & tmask(s);
}

/* ---- FOR fixed-block: FOR_int<T> --------------------------------------- */

/* FOR_int<T>::encodeArray8_int (FOR_integer_template.h:26-81) with
 * write_FOR_int_T (bit_write.h:326-390). */
size_t oracle_for_encode(const void *data, int s, size_t n, uint8_t *out) {
  uint64_t m = ld(data, s, 0), M = m;
  for (size_t i = 1; i < n; i++) {
    uint64_t y = ld(data, s, i);
    if (y > M) M = y;
    if (y < m) m = y;
  }
  unsigned l = (M - m) ? oracle_bits(M - m) : 0;
  if (l > 8u * (unsigned)s) l = 8u * (unsigned)s;
  out[0] = (uint8_t)l;
  if (l == 8u * (unsigned)s) {
    for (size_t i = 0; i < n; i++) { uint64_t y = ld(data, s, i); memcpy(out + 1 + i * (size_t)s, &y, (size_t)s); }
    return 1 + n * (size_t)s;
  }
  memcpy(out + 1, &m, (size_t)s);
  memcpy(out + 1 + s, &M, (size_t)s);
  size_t h = 1 + 2 * (size_t)s;
  if (!l) return h;
  size_t nb = oracle_body_bytes_for(l, n);
  memset(out + h, 0, nb);
  for (size_t i = 0; i < n; i++) put_field(out + h, (uint64_t)i * l, l, (ld(data, s, i) - m) & tmask(s));
  return h + nb;
}

/* FOR_int<T>::decodeArray8 (FOR_integer_template.h:83-112) with
 * read_all_bit_FOR (bit_read.h:1373-1414); strict_raw as for LeCo (:89). */
size_t oracle_for_decode(const uint8_t *in, int s, size_t n, void *out, int strict_raw) {
  unsigned l = in[0];
  unsigned raw_from = strict_raw ? 8u * (unsigned)s : 8u * (unsigned)s - 1;
  if (l >= raw_from) { memcpy(out, in + 1, n * (size_t)s); return n; }
  uint64_t m = rdT(in + 1, s);
  const uint8_t *body = in + 1 + 2 * s;
  for (size_t k = 0; k < n; k++) st(out, s, k, l ? m + get_field(body, (uint64_t)k * l, l) : m);
  return n;
}

/* FOR_int<T>::randomdecodeArray8 (FOR_integer_template.h:218-245), read_FOR_int
 * (bit_read.h:1269-1290). */
uint64_t oracle_for_random(const uint8_t *in, int s, int k) {
  unsigned l = in[0];
  if (l == 8u * (unsigned)s) return rdT(in + 1 + (size_t)k * s, s);
  uint64_t m = rdT(in + 1, s);
  if (!l) return m;
  return (m + get_field(in + 1 + 2 * s, (uint64_t)k * l, l)) & tmask(s);
}

/* ---- Delta fixed-block: Delta_int<T> ----------------------------------- */

/* Delta_int<T>::encodeArray8_int (delta_integer_template.h:26-87).  The
 * reference packs n fields from n-1 deltas (:83), so its last field is read
 * past the end of the delta vector; this restatement writes zero there. */
size_t oracle_delta_encode(const void *data, int s, size_t n, uint8_t *out) {
  uint64_t maxr = 0;
  for (size_t i = 0; i + 1 < n; i++) {
    uint64_t a = ld(data, s, i), b = ld(data, s, i + 1);
    uint64_t r = b > a ? b - a : a - b;
    if (r > maxr) maxr = r;
  }
  unsigned l = maxr ? oracle_bits(maxr) + 1 : 0;
  if (l > 8u * (unsigned)s) l = 8u * (unsigned)s;
  out[0] = (uint8_t)l;
  if (l == 8u * (unsigned)s) {
    for (size_t i = 0; i < n; i++) { uint64_t y = ld(data, s, i); memcpy(out + 1 + i * (size_t)s, &y, (size_t)s); }
    return 1 + n * (size_t)s;
  }
  uint64_t x0 = ld(data, s, 0);
  memcpy(out + 1, &x0, (size_t)s);
  size_t h = 1 + (size_t)s;
  if (!l) return h;
  size_t nb = oracle_body_bytes_signed(l, n);
  memset(out + h, 0, nb);
  for (size_t i = 0; i + 1 < n; i++) {
    uint64_t a = ld(data, s, i), b = ld(data, s, i + 1);
    int pos = b > a;
    put_field(out + h, (uint64_t)i * l, l, sm_field(pos ? b - a : a - b, pos, l));
  }
  return h + nb;
}

/* Delta_int<T>::decodeArray8 (delta_integer_template.h:89-127) with
 * read_all_bit_Delta (bit_read.h:1319-1370).  The reference has no raw path
 * here; raw_ok = 1 decodes a raw block (l == 8s) as raw values instead. */
size_t oracle_delta_decode(const uint8_t *in, int s, size_t n, void *out, int raw_ok) {
  unsigned l = in[0];
  if (l == 127) { st(out, s, 0, rdT(in + 1, s)); return 1; }
  if (l == 126) { st(out, s, 0, rdT(in + 1, s)); st(out, s, 1, rdT(in + 1 + s, s)); return 2; }
  if (raw_ok && l == 8u * (unsigned)s) { memcpy(out, in + 1, n * (size_t)s); return n; }
  uint64_t base = rdT(in + 1, s);
  const uint8_t *body = in + 1 + s;
  st(out, s, 0, base);
  for (size_t k = 1; k < n; k++) {
    if (l) {
      uint64_t f = get_field(body, (uint64_t)(k - 1) * l, l);
      uint64_t mag = f & ((1ull << (l - 1)) - 1);
      base = ((f >> (l - 1)) & 1) ? base + mag : base - mag;
      base &= tmask(s);
    }
    st(out, s, k, base);
  }
  return n;
}

/* Delta_int<T>::randomdecodeArray8 (delta_integer_template.h:132-154),
 * read_Delta_int prefix walk (bit_read.h:1292-1317). */
uint64_t oracle_delta_random(const uint8_t *in, int s, int k) {
  unsigned l = in[0];
  if (l == 8u * (unsigned)s) return rdT(in + 1 + (size_t)k * s, s);
  uint64_t base = rdT(in + 1, s);
  if (!l) return base;
  for (int i = 0; i < k; i++) {
    uint64_t f = get_field(in + 1 + s, (uint64_t)i * l, l);
    uint64_t mag = f & ((1ull << (l - 1)) - 1);
    base = (((f >> (l - 1)) & 1) ? base + mag : base - mag) & tmask(s);
  }
  return base;
}

/* ---- Degree-2 polynomial fixed-block: Leco_int_poly<T,2> --------------- */

/* Leco_int_poly<T,2>::encodeArray8_int (poly_fix_integer_template.h:28-91).
 * No midpoint shift; the residual compares (int64_t)data[i] with the
 * prediction (:42). */
size_t oracle_poly2_encode(const void *data, int s, size_t n, uint8_t *out) {
  double a[3];
  oracle_poly2_fit(data, s, (int)n, a);
  uint64_t maxr = 0;
  for (size_t i = 0; i < n; i++) {
    int64_t pred = x86_f2i(oracle_poly2_eval(a, (double)(int)i));
    int64_t y = (int64_t)ld(data, s, i);
    uint64_t r = (y > pred ? (uint64_t)y - (uint64_t)pred : (uint64_t)pred - (uint64_t)y) & tmask(s);
    if (r > maxr) maxr = r;
  }
  unsigned l = maxr ? oracle_bits(maxr) + 1 : 0;
  if (l > 8u * (unsigned)s) l = 8u * (unsigned)s;
  out[0] = (uint8_t)l;
  if (l == 8u * (unsigned)s) {
    for (size_t i = 0; i < n; i++) { uint64_t y = ld(data, s, i); memcpy(out + 1 + i * (size_t)s, &y, (size_t)s); }
    return 1 + n * (size_t)s;
  }
  memcpy(out + 1, a, 24);
  if (!l) return 25;
  size_t nb = oracle_body_bytes_signed(l, n);
  memset(out + 25, 0, nb);
  for (size_t i = 0; i < n; i++) {
    int64_t pred = x86_f2i(oracle_poly2_eval(a, (double)(int)i));
    int64_t y = (int64_t)ld(data, s, i);
    int pos = y > pred;
    uint64_t r = (pos ? (uint64_t)y - (uint64_t)pred : (uint64_t)pred - (uint64_t)y) & tmask(s);
    put_field(out + 25, (uint64_t)i * l, l, sm_field(r, pos, l));
  }
  return 25 + nb;
}

/* Leco_int_poly<T,2>::decodeArray8 (poly_fix_integer_template.h:93-158) with
 * read_all_bit_fix_poly (bit_read.h:277-330). */
size_t oracle_poly2_decode(const uint8_t *in, int s, size_t n, void *out, int strict_raw) {
  unsigned l = in[0];
  if (l == 127) { st(out, s, 0, rdT(in + 1, s)); return 1; }
  if (l == 126) { st(out, s, 0, rdT(in + 1, s)); st(out, s, 1, rdT(in + 1 + s, s)); return 2; }
  unsigned raw_from = strict_raw ? 8u * (unsigned)s : 8u * (unsigned)s - 1;
  if (l >= raw_from) { memcpy(out, in + 1, n * (size_t)s); return n; }
  double a[3];
  memcpy(a, in + 1, 24);
  for (size_t k = 0; k < n; k++) {
    uint64_t v = (uint64_t)x86_f2i(oracle_poly2_eval(a, (double)(int)k));
    if (l) {
      uint64_t f = get_field(in + 25, (uint64_t)k * l, l);
      uint64_t mag = f & ((1ull << (l - 1)) - 1);
      v = ((f >> (l - 1)) & 1) ? v + mag : v - mag;
    }
    st(out, s, k, v);
  }
  return n;
}

/* Leco_int_poly<T,2>::randomdecodeArray8 (poly_fix_integer_template.h:259-291)
 * with read_bit_fix_int_wo_round_poly (bit_read.h:1201-1232). */
uint64_t oracle_poly2_random(const uint8_t *in, int s, int k) {
  unsigned l = in[0];
  if (l == 8u * (unsigned)s) return rdT(in + 1 + (size_t)k * s, s);
  double a[3];
  memcpy(a, in + 1, 24);
  double p = oracle_poly2_eval(a, (double)k);
  if (!l) return f2T(p, s);
  uint64_t f = get_field(in + 25, (uint64_t)k * l, l);
  uint64_t mag = f & ((1ull << (l - 1)) - 1);
  uint64_t v = (uint64_t)x86_f2i(p);
  v = ((f >> (l - 1)) & 1) ? v + mag : v - mag;
  return v & tmask(s);
}

/* ---- Variable-length segments (Leco_cost_merge_double_wo_round<uint64_t>) -- */

/* newsegment / newsegment_1 / newsegment_2
 * (piecewise_cost_merge_integer_template_double_wo_round.h:134-272): encodes the
 * u64 segment data[start..end] (global indices) as
 * [u32 start][u8 l][f64 theta0][f32 slope][packed], 127 = one value, 126 = two,
 * l == 64 raw.  The prediction is converted to a 128-bit integer (:158). */
size_t oracle_varseg_encode(const uint64_t *array, uint32_t start, uint32_t end, uint8_t *out) {
  memcpy(out, &start, 4);
  if (start == end) { out[4] = 127; memcpy(out + 5, &array[start], 8); return 13; }
  if (end == start + 1) { out[4] = 126; memcpy(out + 5, &array[start], 8); memcpy(out + 13, &array[start + 1], 8); return 21; }
  int length = (int)(end - start + 1);
  double t0, t1;
  oracle_lr_fit(array + start, 8, length, &t0, &t1);
  float slope = (float)t1;
  uint64_t maxr = 0;
  for (uint32_t j = start; j <= end; j++) {
    i128 pred = (i128)(t0 + (double)slope * (double)(j - start));
    i128 y = (i128)array[j];
    uint64_t r = (uint64_t)(y > pred ? y - pred : pred - y);
    if (r > maxr) maxr = r;
  }
  unsigned l = maxr ? oracle_bits(maxr) + 1 : 0;
  if (l >= 64) l = 64;
  out[4] = (uint8_t)l;
  if (l == 64) { memcpy(out + 5, array + start, (size_t)length * 8); return 5 + (size_t)length * 8; }
  memcpy(out + 5, &t0, 8);
  memcpy(out + 13, &slope, 4);
  if (!l) return 17;
  size_t nb = oracle_body_bytes_signed(l, (size_t)length);
  memset(out + 17, 0, nb);
  for (uint32_t j = start; j <= end; j++) {
    i128 pred = (i128)(t0 + (double)slope * (double)(j - start));
    i128 y = (i128)array[j];
    int pos = y > pred;
    uint64_t r = (uint64_t)(pos ? y - pred : pred - y);
    put_field(out + 17, (uint64_t)(j - start) * l, l, sm_field(r, pos, l));
  }
  return 17 + nb;
}

/* One segment of Leco_cost_merge_double_wo_round::decodeArray8 (:581-624) with
 * read_all_bit_fix_wo_round (bit_read.h:505-556), which converts the
 * prediction to uint64_t.  A raw segment is decoded as its own `len` values
 * (the reference copies the whole column length there and returns, :604-607). */
size_t oracle_varseg_decode(const uint8_t *seg, size_t len, uint64_t *out) {
  unsigned l = seg[4];
  if (l == 127) { out[0] = rd64(seg + 5); return 1; }
  if (l == 126) { out[0] = rd64(seg + 5); out[1] = rd64(seg + 13); return 2; }
  if (l > 63) { memcpy(out, seg + 5, len * 8); return len; }
  double t0 = rdf64(seg + 5);
  float t1 = rdf32(seg + 13);
  for (size_t k = 0; k < len; k++) {
    if (!l) { out[k] = x86_f2u(t0 + (double)t1 * (double)k); continue; }
    uint64_t f = get_field(seg + 17, (uint64_t)k * l, l);
    uint64_t mag = f & ((1ull << (l - 1)) - 1);
    uint64_t v = x86_f2u(t0 + (double)k * (double)t1);
    out[k] = ((f >> (l - 1)) & 1) ? v + mag : v - mag;
  }
  return len;
}

/* Leco_cost_merge_double_wo_round::randomdecodeArray8 (:636-698) for the global
 * index g inside this segment; the raw case indexes by the offset inside the
 * segment (the reference uses the global index there, :655-657). */
uint64_t oracle_varseg_random(const uint8_t *seg, uint64_t g) {
  uint32_t start;
  memcpy(&start, seg, 4);
  unsigned l = seg[4];
  uint64_t k = g - start;
  if (l == 64) return rd64(seg + 5 + k * 8);
  if (l == 127) return rd64(seg + 5);
  if (l == 126) return k == 0 ? rd64(seg + 5) : rd64(seg + 13);
  double t0 = rdf64(seg + 5);
  float t1 = rdf32(seg + 13);
  if (!l) return x86_f2u(t0 + (double)t1 * (double)(int)k);
  uint64_t f = get_field(seg + 17, k * l, l);
  uint64_t mag = f & ((1ull << (l - 1)) - 1);
  uint64_t v = (uint64_t)x86_f2i(t0 + (double)(int)k * (double)t1);
  return ((f >> (l - 1)) & 1) ? v + mag : v - mag;
}

/* ---- column drivers (the reference drivers' per-block loops) ------------ */

typedef size_t (*enc_fn)(const void *, int, size_t, uint8_t *);

static enc_fn pick_enc(int codec) {
  switch (codec) {
    case 0: return oracle_leco_encode;
    case 1: return oracle_for_encode;
    case 2: return oracle_delta_encode;
    case 3: return oracle_poly2_encode;
  }
  return 0;
}

/* experiments/leco_int_fix_template.cpp:108-127: blocks of bs values, the last
 * one shorter; images concatenated, offsets[nb] = total bytes. */
size_t oracle_column_encode(int codec, const void *data, int s, size_t n, uint32_t bs, uint8_t *out, uint64_t *offsets) {
  enc_fn f = pick_enc(codec);
  size_t nb = (n + bs - 1) / bs, pos = 0;
  for (size_t b = 0; b < nb; b++) {
    size_t len = n - b * bs < bs ? n - b * bs : bs;
    offsets[b] = pos;
    pos += f((const uint8_t *)data + b * bs * (size_t)s, s, len, out + pos);
  }
  offsets[nb] = pos;
  return pos;
}

/* Bulk decode of a column with the GPU's raw rule (raw iff l == 8s; Delta raw
 * decoded as raw). */
void oracle_column_decode(int codec, const uint8_t *payload, const uint64_t *offsets, int s, size_t n, uint32_t bs, void *out) {
  size_t nb = (n + bs - 1) / bs;
  for (size_t b = 0; b < nb; b++) {
    size_t len = n - b * bs < bs ? n - b * bs : bs;
    uint8_t *o = (uint8_t *)out + b * bs * (size_t)s;
    const uint8_t *in = payload + offsets[b];
    switch (codec) {
      case 0: oracle_leco_decode(in, s, len, o, 1); break;
      case 1: oracle_for_decode(in, s, len, o, 1); break;
      case 2: oracle_delta_decode(in, s, len, o, 1); break;
      case 3: oracle_poly2_decode(in, s, len, o, 1); break;
    }
  }
}

/* Per-index random access over a column (leco_int_fix_template.cpp:189-207). */
void oracle_column_random(int codec, const uint8_t *payload, const uint64_t *offsets, int s, uint32_t bs, const uint64_t *idx, size_t m, void *out) {
  for (size_t i = 0; i < m; i++) {
    const uint8_t *in = payload + offsets[idx[i] / bs];
    int k = (int)(idx[i] % bs);
    uint64_t v = 0;
    switch (codec) {
      case 0: v = oracle_leco_random(in, s, k); break;
      case 1: v = oracle_for_random(in, s, k); break;
      case 2: v = oracle_delta_random(in, s, k); break;
      case 3: v = oracle_poly2_random(in, s, k); break;
    }
    st(out, s, i, v);
  }
}

/* Sum of all decoded values mod 2^64 (the compressed-domain sum's definition). */
uint64_t oracle_column_sum(int codec, const uint8_t *payload, const uint64_t *offsets, int s, size_t n, uint32_t bs, void *scratch) {
  oracle_column_decode(codec, payload, offsets, s, n, bs, scratch);
  uint64_t acc = 0;
  for (size_t i = 0; i < n; i++) acc += ld(scratch, s, i);
  return acc;
}

/* ---- predicate pushdown ------------------------------------------------- */

/* (int)x as x86-64 compiles it (32-bit CVTTSD2SI): NaN and values outside the
 * int range give INT_MIN.  The filters store their FP64 index thresholds in
 * int (piecewise_fix_integer_template.h:226,275-276). */
static int32_t x86_f2i32(double x) {
  if (x > -2147483649.0 && x < 2147483648.0) return (int32_t)x;
  return INT32_MIN;
}
/* std::max(a, b) = (a < b) ? b : a and std::min(a, b) = (b < a) ? b : a, as
 * the filters call them (a NaN first argument passes through). */
static double std_max(double a, double b) { return a < b ? b : a; }
static double std_min(double a, double b) { return b < a ? b : a; }

/* Comparisons of a decoded value with a filter bound of type T: for T =
 * uint64_t the reference compares int64_t with T, i.e. unsigned; for T =
 * uint32_t the bound is promoted to int64_t and the comparison is signed
 * (bit_read.h:421,477; piecewise_fix_integer_template.h:241,286). */
static int cmp_gt(uint64_t v, uint64_t f, int s) { return s == 8 ? v > f : (int64_t)v > (int64_t)f; }
static int cmp_lt(uint64_t v, uint64_t f, int s) { return s == 8 ? v < f : (int64_t)v < (int64_t)f; }

/* Value k of a packed LeCo block as the filter readers compute it:
 * (long long)(theta0 + k*theta1) minus or plus the field's magnitude, in
 * wrapping 64-bit arithmetic (bit_read.h:409-420,465-476); l == 0: the
 * prediction alone (piecewise_fix_integer_template.h:240,285). */
static uint64_t leco_filter_value(const uint8_t *body, unsigned l, double t0, double t1, int64_t k) {
  uint64_t v = (uint64_t)x86_f2i(t0 + (double)k * t1);
  if (!l) return v;
  uint64_t f = get_field(body, (uint64_t)k * l, l);
  uint64_t mag = f & ((1ull << (l - 1)) - 1);
  return ((f >> (l - 1)) & 1) ? v + mag : v - mag;
}

/* 1L << (l-1), the model's residual bound (:221-224, :270-273). */
static int64_t delta_interval(unsigned l) { return l ? (int64_t)1 << (l - 1) : 0; }

/* (double)(filter + c) for a bound of type T plus an int64_t offset c: T =
 * uint64_t wraps modulo 2^64 and converts as unsigned; T = uint32_t computes in
 * int64_t (:226, :275-276).  plus_one adds the int 1 first, in T (:226). */
static double bound_to_double(uint64_t filter, int plus_one, int64_t c, int s) {
  if (s == 8) return (double)(filter + (uint64_t)plus_one + (uint64_t)c);
  uint32_t f = (uint32_t)filter + (uint32_t)plus_one;
  return (double)((int64_t)f + c);
}

/* Leco_int<T>::filter_range (piecewise_fix_integer_template.h:206-252) with
 * read_all_bit_fix_range (bit_read.h:388-445): the indices block_start + k of
 * the values above `filter`, scanned from the model's threshold
 * thre = (int)max((filter + 1 - 2^(l-1) - theta0) / theta1, 0).  A raw block
 * (l == 8s), which the reference does not recognise here (its result would
 * come from shifts by the type width), is scanned as its stored values.
 * Returns the count. */
size_t oracle_leco_filter(const uint8_t *in, int s, size_t n, uint64_t filter, uint32_t block_start, uint32_t *out) {
  unsigned l = in[0];
  size_t c = 0;
  filter &= tmask(s);
  if (l == 8u * (unsigned)s) {
    for (size_t k = 0; k < n; k++)
      if (rdT(in + 1 + k * (size_t)s, s) > filter) out[c++] = block_start + (uint32_t)k;
    return c;
  }
  double t0 = rdf64(in + 1), t1 = rdf64(in + 9);
  int32_t thre = x86_f2i32(std_max((bound_to_double(filter, 1, -delta_interval(l), s) - t0) / t1, 0.));
  if ((uint64_t)(int64_t)thre >= n) return 0; /* :227 compares int with size_t */
  for (size_t k = (size_t)thre; k < n; k++)
    if (cmp_gt(leco_filter_value(in + 17, l, t0, t1, (int64_t)k), filter, s)) out[c++] = block_start + (uint32_t)k;
  return c;
}

/* Leco_int<T>::filter_range_close (piecewise_fix_integer_template.h:254-303)
 * with read_all_bit_fix_range_close (bit_read.h:447-502): for the windows
 * (filter1 + p*base, filter2 + p*base), p = 0, 1, ... (bounds wrap in T), the
 * indices whose value lies strictly inside, scanned over the model's index range
 * [thre1, thre2) per window ([thre1, thre2] for l == 0, :281) until
 * thre1 >= length or thre2 <= 0.
 * overwrite = 1 reproduces the reference's output pointer exactly: for l > 0
 * every window's indices are written from out[0] again (the reader is passed
 * `out`, not the advanced position, :280), so earlier windows' indices are
 * overwritten; overwrite = 0 writes them one after another.  The count is the
 * same.  Raw blocks: every stored value is counted once when it lies in some
 * window.  max_periods bounds the window loop (0 = unbounded); returns the
 * count, or SIZE_MAX when the bound was reached. */
size_t oracle_leco_filter_close(const uint8_t *in, int s, size_t n, uint64_t filter1, uint64_t filter2, int32_t base,
                                uint32_t block_start, uint32_t *out, int overwrite, uint64_t max_periods) {
  unsigned l = in[0];
  size_t c = 0;
  const uint64_t mask = tmask(s);
  filter1 &= mask;
  filter2 &= mask;
  if (l == 8u * (unsigned)s) {
    const uint64_t b = (uint64_t)(int64_t)base & mask;
    for (size_t k = 0; k < n; k++) {
      uint64_t v = rdT(in + 1 + k * (size_t)s, s);
      if (v <= filter1 || filter2 <= filter1 || b == 0) continue;
      uint64_t m = (v - filter1 - 1) % b; /* the largest window start below v is v - m - 1 */
      if (m + 1 < filter2 - filter1) out[c++] = block_start + (uint32_t)k;
    }
    return c;
  }
  double t0 = rdf64(in + 1), t1 = rdf64(in + 9);
  const int64_t di = delta_interval(l);
  const uint64_t step = (uint64_t)(int64_t)base & mask; /* filter += base in T (:290-291) */
  uint64_t p = 0;
  for (;;) {
    int32_t thre1 = x86_f2i32(std_max((bound_to_double(filter1, 0, -di, s) - t0) / t1 - 1, 0.));
    int32_t thre2 = x86_f2i32(std_min((bound_to_double(filter2, 0, di, s) - t0) / t1 + 1, (double)n));
    if (!((uint64_t)(int64_t)thre1 < n && thre2 > 0)) break;
    if (max_periods && p == max_periods) return (size_t)-1;
    uint32_t *o = (overwrite && l) ? out : out + c;
    size_t pc = 0;
    int64_t hi = l ? (int64_t)thre2 : (int64_t)thre2 + 1;
    for (int64_t k = thre1; k < hi; k++) {
      uint64_t v = leco_filter_value(in + 17, l, t0, t1, k);
      if (cmp_gt(v, filter1, s) && cmp_lt(v, filter2, s)) o[pc++] = block_start + (uint32_t)k;
    }
    c += pc;
    filter1 = (filter1 + step) & mask;
    filter2 = (filter2 + step) & mask;
    p++;
  }
  return c;
}

/* FOR_int<T>::filter_range (FOR_integer_template.h:115-160) with
 * filter_read_all_bit_FOR (bit_read.h:1417-1459): values above `filter`; the
 * header maximum rejects a block unread (:143).  Raw iff l == 8s (the
 * reference's `l >= 8s-1` test reads an l == 8s-1 packed block as raw). */
size_t oracle_for_filter(const uint8_t *in, int s, size_t n, uint64_t filter, uint32_t block_start, uint32_t *out) {
  unsigned l = in[0];
  size_t c = 0;
  filter &= tmask(s);
  if (l == 8u * (unsigned)s) {
    for (size_t k = 0; k < n; k++)
      if (rdT(in + 1 + k * (size_t)s, s) > filter) out[c++] = block_start + (uint32_t)k;
    return c;
  }
  uint64_t m = rdT(in + 1, s), M = rdT(in + 1 + s, s);
  if (M <= filter) return 0;
  for (size_t k = 0; k < n; k++) {
    uint64_t v = l ? (m + get_field(in + 1 + 2 * s, (uint64_t)k * l, l)) & tmask(s) : m;
    if (v > filter) out[c++] = block_start + (uint32_t)k;
  }
  return c;
}

/* FOR_int<T>::filter_range_close (FOR_integer_template.h:166-215) with
 * filter_read_all_bit_FOR_close (bit_read.h:1462-1505): values v with
 * filter1 < v % base < filter2 (base converted to T). */
size_t oracle_for_filter_close(const uint8_t *in, int s, size_t n, uint64_t filter1, uint64_t filter2, int32_t base,
                               uint32_t block_start, uint32_t *out) {
  unsigned l = in[0];
  size_t c = 0;
  const uint64_t mask = tmask(s), b = (uint64_t)(int64_t)base & mask;
  filter1 &= mask;
  filter2 &= mask;
  if (b == 0) return 0;
  int raw = l == 8u * (unsigned)s;
  uint64_t m = raw ? 0 : rdT(in + 1, s);
  for (size_t k = 0; k < n; k++) {
    uint64_t v = raw ? rdT(in + 1 + k * (size_t)s, s) : (l ? (m + get_field(in + 1 + 2 * s, (uint64_t)k * l, l)) & mask : m);
    uint64_t r = v % b;
    if (r > filter1 && r < filter2) out[c++] = block_start + (uint32_t)k;
  }
  return c;
}

/* Per-block minimum and maximum of a column's decoded values (the filter
 * experiments' zone map, experiments/leco_int_fix_template.cpp:219-239). */
void oracle_column_zonemap(int codec, const uint8_t *payload, const uint64_t *offsets, int s, size_t n, uint32_t bs,
                           void *scratch, uint64_t *zmin, uint64_t *zmax) {
  oracle_column_decode(codec, payload, offsets, s, n, bs, scratch);
  size_t nb = (n + bs - 1) / bs;
  for (size_t b = 0; b < nb; b++) {
    size_t len = n - b * bs < bs ? n - b * bs : bs;
    uint64_t lo = ~0ull, hi = 0;
    for (size_t k = 0; k < len; k++) {
      uint64_t v = ld(scratch, s, b * bs + k);
      if (v < lo) lo = v;
      if (v > hi) hi = v;
    }
    zmin[b] = lo;
    zmax[b] = hi;
  }
}

/* The filter experiment's loop (experiments/leco_int_fix_template.cpp:244-256,
 * FOR_int_fix_template.cpp:254-266): blocks in order, results appended; with a
 * zone map, blocks whose maximum is <= filter are skipped.  Returns the count. */
size_t oracle_column_filter(int codec, const uint8_t *payload, const uint64_t *offsets, int s, size_t n, uint32_t bs,
                            uint64_t filter, const uint64_t *zmax, uint32_t *out) {
  size_t nb = (n + bs - 1) / bs, c = 0;
  for (size_t b = 0; b < nb; b++) {
    if (zmax && zmax[b] <= filter) continue;
    size_t len = n - b * bs < bs ? n - b * bs : bs;
    const uint8_t *in = payload + offsets[b];
    uint32_t start = (uint32_t)(b * bs);
    c += codec == 0 ? oracle_leco_filter(in, s, len, filter, start, out + c) : oracle_for_filter(in, s, len, filter, start, out + c);
  }
  return c;
}

/* Window start of one block in the LeCo close-range experiment
 * (experiments/leco_int_fix_template.cpp:299-304): the first
 * filter1 + j*base at or above the block minimum, one window earlier when the
 * minimum itself lies inside a window; all in T and FP64 as written there
 * (base is the driver's T). */
void oracle_close_window_start(uint64_t zmin, uint64_t filter1, uint64_t filter2, uint64_t base, int s,
                               uint64_t *f1_out, uint64_t *f2_out) {
  const uint64_t mask = tmask(s);
  double q = __builtin_ceil((double)((zmin - filter1) & mask) / (double)base);
  uint64_t a = f2T(q * (double)base + (double)filter1, s);
  uint64_t b = f2T(q * (double)base + (double)filter2, s);
  uint64_t r = zmin % base;
  if (r < filter2 && r > filter1) {
    a = (a - base) & mask;
    b = (b - base) & mask;
  }
  *f1_out = a;
  *f2_out = b;
}

/* The close-range experiment's loop (leco_int_fix_template.cpp:290-322 for
 * LeCo, FOR_int_fix_template.cpp:303-322 for FOR): LeCo blocks get their own
 * window start from the zone-map minimum (or filter1/filter2 as given when zmin
 * is NULL); FOR blocks take filter1, filter2, base as given.  base is passed to
 * the codec as int (:310).  overwrite as in oracle_leco_filter_close.  Returns
 * the count, or SIZE_MAX when a block reached max_periods windows. */
size_t oracle_column_filter_close(int codec, const uint8_t *payload, const uint64_t *offsets, int s, size_t n, uint32_t bs,
                                  uint64_t filter1, uint64_t filter2, uint64_t base, const uint64_t *zmin, uint32_t *out,
                                  int overwrite, uint64_t max_periods) {
  size_t nb = (n + bs - 1) / bs, c = 0;
  for (size_t b = 0; b < nb; b++) {
    size_t len = n - b * bs < bs ? n - b * bs : bs;
    const uint8_t *in = payload + offsets[b];
    uint32_t start = (uint32_t)(b * bs);
    if (codec == 0) {
      uint64_t f1 = filter1, f2 = filter2;
      if (zmin) oracle_close_window_start(zmin[b], filter1, filter2, base, s, &f1, &f2);
      size_t k = oracle_leco_filter_close(in, s, len, f1, f2, (int32_t)base, start, out + c, overwrite, max_periods);
      if (k == (size_t)-1) return k;
      c += k;
    } else {
      c += oracle_for_filter_close(in, s, len, filter1, filter2, (int32_t)base, start, out + c);
    }
  }
  return c;
}

/* ---- legacy u32 format: piecewise_fix_op_max ------------------------------ */

/* piecewise_fix_op_max::encodeArray8 (piecewise_fix_op_minimize_maxerror.h:45-119):
 * lr_int fit (lr.h:89-111, the same sums as lr_int_T), slope stored as float, the
 * midpoint shift in int arithmetic, int residuals against (long long)(theta0 +
 * theta1*i), width bits(max |r|) + 1; header [u8 l][f64 theta0][f32 theta1]; body
 * packed with write_delta_T (bit_write.h:186-245, pad (32-l)/8 bytes) for l <= 30,
 * the values as u32 (write_delta_default, :395-410) for l >= 31.
 * diff_plus / diff_minus (nullable, n bytes each) receive the encoder's
 * mul_add_diff_set / mul_add_diff_set_minus flags (:79-84): where the prediction
 * accumulated by addition is below / above the multiplied one.  Returns bytes. */
size_t oracle_legacy_encode(const uint32_t *in, size_t n, uint8_t *out, uint8_t *diff_plus, uint8_t *diff_minus) {
  double t0, t1d;
  oracle_lr_fit(in, 4, (int)n, &t0, &t1d);
  const float t1 = (float)t1d;
  int32_t mx = INT32_MIN, mn = INT32_MAX;
  for (size_t i = 0; i < n; i++) {
    int32_t d = (int32_t)((int64_t)in[i] - x86_f2i(t0 + (double)t1 * (double)i));
    if (d > mx) mx = d;
    if (d < mn) mn = d;
  }
  t0 += (double)(int32_t)((uint32_t)mx + (uint32_t)mn) / 2.0;
  double pred = t0;
  uint32_t maxe = 0;
  int32_t *delta = (int32_t *)__builtin_alloca(n * sizeof(int32_t) + 4);
  for (size_t i = 0; i < n; i++) {
    const int64_t pm = x86_f2i(t0 + (double)t1 * (double)i), pa = x86_f2i(pred);
    if (diff_plus) diff_plus[i] = pm > pa;
    if (diff_minus) diff_minus[i] = pm < pa;
    pred += (double)t1;
    const int32_t d = (int32_t)((int64_t)in[i] - pm);
    delta[i] = d;
    /* abs(INT_MIN) stays INT_MIN on x86 and fails the reference's `> max_error` */
    const uint32_t a = d == INT32_MIN ? 0u : d < 0 ? (uint32_t)(-(int64_t)d) : (uint32_t)d;
    if (a > maxe) maxe = a;
  }
  const unsigned l = maxe ? (unsigned)oracle_bits(maxe) + 1 : 0;
  out[0] = (uint8_t)l;
  memcpy(out + 1, &t0, 8);
  memcpy(out + 9, &t1, 4);
  if (!l) return 13;
  if (l >= 31) {
    memcpy(out + 13, in, n * 4);
    return 13 + n * 4;
  }
  const size_t nb = oracle_body_bytes_for(l, n); /* end + 1 + (32-l)/8 */
  uint8_t *body = out + 13;
  memset(body, 0, nb);
  for (size_t i = 0; i < n; i++) {
    const int32_t d = delta[i];
    const uint64_t mag = d <= 0 ? (uint64_t)(-(int64_t)d) : (uint64_t)d;
    put_field(body, (uint64_t)i * l, l, (mag & ((1ull << (l - 1)) - 1)) | ((uint64_t)(d > 0) << (l - 1)));
  }
  return 13 + nb;
}

/* Bulk decode.  add_pred = 1: piecewise_fix_op_max::decodeArray8 (:121-158) as
 * written -- the prediction accumulated by repeated addition (read_all_bit_fix_add,
 * bit_read.h:559-605; the l == 0 loop :148-153), which the reference's drivers then
 * correct with the encoder's difference lists (experiments/fix_int.cpp:110-117);
 * add_pred = 0: the multiplied prediction the encoder and the random access use,
 * i.e. the stored values. */
void oracle_legacy_decode(const uint8_t *in, size_t n, uint32_t *out, int add_pred) {
  const unsigned l = in[0];
  double t0;
  float t1;
  memcpy(&t0, in + 1, 8);
  memcpy(&t1, in + 9, 4);
  if (l >= 31) {
    memcpy(out, in + 13, n * 4);
    return;
  }
  double pred = t0;
  for (size_t k = 0; k < n; k++) {
    int64_t p = add_pred ? x86_f2i(pred) : x86_f2i(t0 + (double)t1 * (double)k);
    pred += (double)t1;
    if (l) {
      const uint64_t f = get_field(in + 13, (uint64_t)k * l, l);
      const int64_t mag = (int64_t)(f & ((1ull << (l - 1)) - 1));
      p = ((f >> (l - 1)) & 1) ? p + mag : p - mag;
    }
    out[k] = (uint32_t)p;
  }
}

/* piecewise_fix_op_max::randomdecodeArray8 (:160-186) with read_bit_fix_T
 * (bit_read.h:1107-1133) / read_bit_default (:61-74). */
uint32_t oracle_legacy_random(const uint8_t *in, int k) {
  const unsigned l = in[0];
  double t0;
  float t1;
  memcpy(&t0, in + 1, 8);
  memcpy(&t1, in + 9, 4);
  if (l >= 31) {
    uint32_t v;
    memcpy(&v, in + 13 + 4 * (size_t)k, 4);
    return v;
  }
  const int64_t p = x86_f2i(t0 + (double)k * (double)t1);
  if (!l) return (uint32_t)p;
  const uint64_t f = get_field(in + 13, (uint64_t)k * l, l);
  const int64_t mag = (int64_t)(f & ((1ull << (l - 1)) - 1));
  return (uint32_t)(((f >> (l - 1)) & 1) ? p + mag : p - mag);
}
