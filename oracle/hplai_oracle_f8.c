/*
 * hplai_oracle_f8.c -- CPU oracle for the precision form's e4m3 panels.
 *
 * TEST INFRASTRUCTURE ONLY (see hplai_oracle.c): linked into liboracle.so,
 * never into the product.
 *
 * The precision form has no counterpart in the reference; its down-cast
 * generalises convert_left_panels / convert_right_panels
 * (panel_trf.hpp:173-233), which multiply an FP32 panel by one factor and
 * round it to the low format, to one power-of-two factor per 128 rows and the
 * OCP FP8 e4m3 format (1 sign bit, 4 exponent bits with bias 7, 3 mantissa
 * bits, subnormals with quantum 2^-9, largest finite 448, no infinities).
 * The rounding is restated here from that definition: round to nearest,
 * ties to even, saturating at 448.
 */
#include <stdint.h>
#include <math.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* e4m3 encoding of x, round to nearest even, finite values saturate at 448. */
ORC_EXPORT uint8_t orc_e4m3_rn(float x)
{
	if (x != x) return 0x7F;
	const uint8_t sign = signbit(x) ? 0x80 : 0x00;
	double a = fabs((double)x);
	if (a == 0.0) return sign;
	int e2;
	frexp(a, &e2);                 /* a = m 2^e2, m in [0.5, 1): a in [2^(e2-1), 2^e2) */
	int e = e2 - 1;                /* floor(log2 a) */
	if (e < -6) e = -6;            /* subnormal range shares the quantum of 2^-6 */
	const double quantum = ldexp(1.0, e - 3);
	double q = nearbyint(a / quantum);   /* a / quantum is exact (power of two), default mode RNE */
	double v = q * quantum;
	if (v > 448.0) v = 448.0;
	/* encode v exactly */
	if (v < ldexp(1.0, -6)) {
		const int mant = (int)(v / ldexp(1.0, -9));
		return (uint8_t)(sign | mant);
	}
	frexp(v, &e2);
	e = e2 - 1;
	const int mant = (int)(v / ldexp(1.0, e - 3)) - 8;
	return (uint8_t)(sign | ((e + 7) << 3) | mant);
}

ORC_EXPORT float orc_e4m3_to_f32(uint8_t b)
{
	const int s = b >> 7, ex = (b >> 3) & 15, m = b & 7;
	if (ex == 15 && m == 7) return NAN;
	const double v = ex == 0 ? ldexp((double)m, -9) : ldexp(8.0 + m, ex - 10);
	return (float)(s ? -v : v);
}

/* Per-128-row power-of-two factor and e4m3 copy (the precision form's
 * down-cast).  X element (r, p) at src[r + p*lds] (col_major) or
 * src[p + r*lds].  dst row r at dst + r*ld8, bytes k..ld8 zero. */
ORC_EXPORT void orc_quantize_e4m3(int rows, int k, const float *src, int64_t lds, int col_major, uint8_t *dst,
	int64_t ld8, float *scale)
{
	for (int r0 = 0; r0 < rows; r0 += 128) {
		const int r1 = r0 + 128 < rows ? r0 + 128 : rows;
		float amax = 0.f;
		for (int r = r0; r < r1; ++r)
			for (int p = 0; p < k; ++p) {
				const float v = fabsf(col_major ? src[r + (int64_t)p * lds] : src[p + (int64_t)r * lds]);
				if (v > amax) amax = v;
			}
		int e = 0;
		if (amax > 0.f) frexpf(amax / 448.f, &e);
		const float inv = ldexpf(1.f, -e);
		scale[r0 / 128] = ldexpf(1.f, e);
		for (int r = r0; r < r1; ++r) {
			for (int p = 0; p < k; ++p) {
				const float v = col_major ? src[r + (int64_t)p * lds] : src[p + (int64_t)r * lds];
				dst[(int64_t)r * ld8 + p] = orc_e4m3_rn(v * inv);
			}
			for (int64_t p = k; p < ld8; ++p) dst[(int64_t)r * ld8 + p] = 0;
		}
	}
}

/* C -= diag(sl) L8 U8^T diag(su) with the products summed in FP64 (the
 * e4m3 products are exact; the device sums them in FP32). */
ORC_EXPORT void orc_f8gemm_minus(int m, int n, int k, const uint8_t *l8, int64_t ldl, const float *sl,
	const uint8_t *u8, int64_t ldu, const float *su, float *c, int64_t ldc)
{
	for (int j = 0; j < n; ++j)
		for (int i = 0; i < m; ++i) {
			double s = 0.0;
			for (int p = 0; p < k; ++p)
				s += (double)orc_e4m3_to_f32(l8[(int64_t)i * ldl + p]) * orc_e4m3_to_f32(u8[(int64_t)j * ldu + p]);
			s *= (double)sl[i / 128] * (double)su[j / 128];
			c[i + (int64_t)j * ldc] = (float)((double)c[i + (int64_t)j * ldc] - s);
		}
}
