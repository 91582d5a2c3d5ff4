// Constants and inline device helpers of the EMC iteration for sm_100a (B200).
//
// Layout conventions (all in HBM, owned by the context in emc_api.cu):
//   R        = num_modes * num_rot orientations, processed in tiles of
//              TILE = 32 * LW (one warp; each lane owns LW consecutive
//              orientations, so a row of a tile is one vector load per lane);
//              RT = ceil(R / TILE) tiles, orientation
//              r = tile * TILE + lane * LW + k, r -> (rotation r / M, mode r % M)
//              as in dragonfly/src/max_prob.c:80-85.
//   logW     [RT][P+1][TILE] float log of the slice W_r[p], pixel-major inside
//                                a tile so that every photon gather reads one
//                                coalesced row (4 * TILE bytes); row P is all
//                                zero (target of padding words).
//   pval     [RT][Nc][TILE] double log-likelihood of (orientation, frame)
//                                pairs of the current frame chunk.
//   tmax/targ [RT][Nc]           per (tile, frame) maximum pval and its lowest r.
//   Pst      [RT][Nc+1][TILE] float normalised probability of kept pairs; the
//                                sign carries the reference's PROB_MIN gate:
//                                P > 1e-6 stored as +P, kept but <= 1e-6 as -P,
//                                pruned 0; row Nc is all zero.
//   T        [RT][P][TILE] float  photon tomograms sum_d P_dr * K_d[p].
//   accum    [M*V] double2       (model2 sum, weight) merge accumulators.
// Photon lists: per frame (E-step) or per pixel (M-step) a segment of
// count-1 photons followed by a segment of multi-photon words, each padded to
// a multiple of 8 with words that point at the zero row. Count-1 words hold
// the pixel (E-step) or chunk-local frame (M-step); multi words hold that
// index in the low 22 bits and the count in the high 10 bits (counts above
// 1023 are split over several words; every use is linear in the count).
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

// Orientations per lane: 4 makes every photon gather one 16-byte load per
// lane (a 512-byte row per warp), which moves four times the bytes per load
// instruction and per photon-word fetch of a one-orientation lane.
#ifndef DFG_LANE_W
#define DFG_LANE_W 4
#endif

namespace dfg {

constexpr int LW = DFG_LANE_W;
static_assert(LW == 1 || LW == 2 || LW == 4, "lane width must be 1, 2 or 4");
constexpr int TILE = 32 * LW;
constexpr int IDX_BITS = 22;
constexpr uint32_t IDX_MASK = (1u << IDX_BITS) - 1u;
constexpr uint32_t MAX_COUNT = (1u << (32 - IDX_BITS)) - 1u;
constexpr double PROB_MIN = 1.e-6;          // dragonfly/src/max_internal.h:6
constexpr double PDIFF_THRESH = 14.;        // dragonfly/src/max_internal.h:7
constexpr double MAX_EXP_START = -1.e100;   // dragonfly/src/max_internal.h:8
constexpr int PB = 64;                      // pixels per block in slice / merge kernels
constexpr int MAX_MODES = 16;
constexpr unsigned FULL = 0xffffffffu;

// FP64 arithmetic in the reference's operation order: these intrinsics are
// never contracted into fused multiply-adds, so geometry (cell index, OOB
// test, interpolation weights) is bit-identical to the C engine.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Rotation matrix of a quaternion (dragonfly/src/model.c:759-786), row-major.
__device__ inline void rot_from_quat(const double *q, double *rot) {
	double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
	double q01 = dmul(q0, q1), q02 = dmul(q0, q2), q03 = dmul(q0, q3);
	double q11 = dmul(q1, q1), q12 = dmul(q1, q2), q13 = dmul(q1, q3);
	double q22 = dmul(q2, q2), q23 = dmul(q2, q3), q33 = dmul(q3, q3);
	rot[0] = dsub(1., dmul(2., dadd(q22, q33)));
	rot[1] = dmul(2., dadd(q12, q03));
	rot[2] = dmul(2., dsub(q13, q02));
	rot[3] = dmul(2., dsub(q12, q03));
	rot[4] = dsub(1., dmul(2., dadd(q11, q33)));
	rot[5] = dmul(2., dadd(q01, q23));
	rot[6] = dmul(2., dadd(q02, q13));
	rot[7] = dmul(2., dsub(q23, q01));
	rot[8] = dsub(1., dmul(2., dadd(q11, q22)));
}

// Trilinear cell of a detector pixel rotated into the model grid, computed as
// slice_gen3d / slice_merge3d do (model.c:19-44, 177-201): position
// sum_j rot[i][j] q_j + center, integer part by truncation toward zero,
// in bounds iff 0 <= x <= size-2 on every axis.
struct Cell {
	long long i000;  // x*S*S + y*S + z
	double fx, fy, fz;
	bool ok;
};

__device__ __forceinline__ Cell locate(const double *rot, double qx, double qy, double qz, double center,
                                       long long S) {
	Cell c;
	double px = dadd(dadd(dadd(dmul(rot[0], qx), dmul(rot[1], qy)), dmul(rot[2], qz)), center);
	double py = dadd(dadd(dadd(dmul(rot[3], qx), dmul(rot[4], qy)), dmul(rot[5], qz)), center);
	double pz = dadd(dadd(dadd(dmul(rot[6], qx), dmul(rot[7], qy)), dmul(rot[8], qz)), center);
	long long x = (long long)px, y = (long long)py, z = (long long)pz;
	c.ok = !(x < 0 || x > S - 2 || y < 0 || y > S - 2 || z < 0 || z > S - 2);
	c.fx = dsub(px, (double)x);
	c.fy = dsub(py, (double)y);
	c.fz = dsub(pz, (double)z);
	c.i000 = c.ok ? (x * S + y) * S + z : 0;
	return c;
}

// The 8 corner weights in the reference's order (000, 001, 010, 011, 100, ...).
__device__ __forceinline__ void corner_weights(const Cell &c, double *w) {
	double cx = dsub(1., c.fx), cy = dsub(1., c.fy), cz = dsub(1., c.fz);
	double cxcy = dmul(cx, cy), cxfy = dmul(cx, c.fy), fxcy = dmul(c.fx, cy), fxfy = dmul(c.fx, c.fy);
	w[0] = dmul(cxcy, cz); w[1] = dmul(cxcy, c.fz);
	w[2] = dmul(cxfy, cz); w[3] = dmul(cxfy, c.fz);
	w[4] = dmul(fxcy, cz); w[5] = dmul(fxcy, c.fz);
	w[6] = dmul(fxfy, cz); w[7] = dmul(fxfy, c.fz);
}

__device__ __forceinline__ void corner_offsets(long long S, long long *o) {
	// +z, +y, +x neighbours; (x+1) % S == x+1 inside bounds
	o[0] = 0; o[1] = 1; o[2] = S; o[3] = S + 1;
	o[4] = S * S; o[5] = S * S + 1; o[6] = S * S + S; o[7] = S * S + S + 1;
}

// W = corr * sum_k w_k m_k, summed left to right; DBL_MIN outside the model
// (model.c:33-57).
template <typename MT>
__device__ __forceinline__ double interp(const Cell &c, const MT *__restrict__ m, long long S, double corr) {
	if (!c.ok)
		return DBL_MIN;
	double w[8];
	long long o[8];
	corner_weights(c, w);
	corner_offsets(S, o);
	double v = dmul(w[0], (double)__ldg(m + c.i000));
#pragma unroll
	for (int k = 1; k < 8; ++k)
		v = dadd(v, dmul(w[k], (double)__ldg(m + c.i000 + o[k])));
	return dmul(v, corr);
}

// Model types (enum model_type, model.h:13): a volume sampled trilinearly at
// quaternion-rotated pixel positions, a stack of 2-D images sampled
// bilinearly at in-plane-rotated positions (orientation = angle), or an RZ
// image (orientation = (phi, beta)).
enum ModelType { MT_3D = 0, MT_2D = 1, MT_RZ = 2 };

// Bilinear cell in a 2-D image: integer part by truncation toward zero, in
// bounds iff 0 <= x, y <= size-2 (model.c:85-99, 133-146, 280-290).
struct Cell2 {
	long long i00;  // x*S + y
	double fx, fy;
	bool ok;
};

__device__ __forceinline__ Cell2 cell2_at(double px, double py, long long S) {
	Cell2 c;
	const long long x = (long long)px, y = (long long)py;
	c.ok = !(x < 0 || x > S - 2 || y < 0 || y > S - 2);
	c.fx = dsub(px, (double)x);
	c.fy = dsub(py, (double)y);
	c.i00 = c.ok ? x * S + y : 0;
	return c;
}

// slice_gen2d / slice_merge2d (model.c:65-99, 254-280): the pixel's (qx, qy)
// rotated by rot = [[c, -s], [s, c]] (make_rot_angle, model.c:788-795; c and
// s come from the host's libm), plus the center.
__device__ __forceinline__ Cell2 locate2d(const double *cs, double qx, double qy, double center, long long S) {
	const double px = dadd(dadd(dmul(cs[0], qx), dmul(-cs[1], qy)), center);
	const double py = dadd(dadd(dmul(cs[1], qx), dmul(cs[0], qy)), center);
	return cell2_at(px, py, S);
}

// slice_genrz / slice_mergerz (model.c:106-150, 305-340): g = (cos phi,
// sin phi, cos beta, sin beta, detd). The pixel is projected with
// fac = detd^2 + qx^2 + qy^2, rotated by phi in the detector plane, then the
// (y, z) components by beta; the image coordinates are the radius in the
// (x, z) plane and y, scaled by the center.
__device__ __forceinline__ Cell2 locate_rz(const double *g, double qx, double qy, double center, long long S) {
	const double detd = g[4];
	const double fac = dadd(dmul(detd, detd), dadd(dmul(qx, qx), dmul(qy, qy)));
	const double q0 = __ddiv_rn(dadd(dmul(qx, g[0]), dmul(qy, -g[1])), fac);
	const double q1 = __ddiv_rn(dadd(dmul(qx, g[1]), dmul(qy, g[0])), fac);
	const double q2 = dsub(__ddiv_rn(detd, fac), 1.);
	const double b1 = dadd(dmul(q1, g[2]), dmul(q2, -g[3]));
	const double b2 = dadd(dmul(q1, g[3]), dmul(q2, g[2]));
	const double px = dmul(center, dadd(1., __dsqrt_rn(dadd(dmul(q0, q0), dmul(b2, b2)))));
	const double py = dmul(center, dadd(1., b1));
	return cell2_at(px, py, S);
}

// The 4 corner weights in the reference's order (00, 01, 10, 11).
__device__ __forceinline__ void corner_weights2(const Cell2 &c, double *w) {
	const double cx = dsub(1., c.fx), cy = dsub(1., c.fy);
	w[0] = dmul(cx, cy);
	w[1] = dmul(cx, c.fy);
	w[2] = dmul(c.fx, cy);
	w[3] = dmul(c.fx, c.fy);
}

// W = corr * sum_k w_k m_k, summed left to right; DBL_MIN outside the image
// and where W <= 0 (model.c:88-99, 136-149).
template <typename MT>
__device__ __forceinline__ double interp2(const Cell2 &c, const MT *__restrict__ m, long long S, double corr) {
	if (!c.ok)
		return DBL_MIN;
	double w[4];
	corner_weights2(c, w);
	double v = dmul(w[0], (double)__ldg(m + c.i00));
	v = dadd(v, dmul(w[1], (double)__ldg(m + c.i00 + 1)));
	v = dadd(v, dmul(w[2], (double)__ldg(m + c.i00 + S)));
	v = dadd(v, dmul(w[3], (double)__ldg(m + c.i00 + S + 1)));
	v = dmul(v, corr);
	return v <= 0. ? DBL_MIN : v;
}

// Orientation parameters of orientation qi staged in rot[9]: the rotation
// matrix of quaternion geo[qi * 5 ..] (3-D), or (cos, sin) of its angle from
// the host-made table geo[qi * 2 ..] (2-D).
template <int GEO>
__device__ __forceinline__ void geo_setup(const double *__restrict__ geo, int qi, double *rot) {
	if constexpr (GEO == MT_3D) {
		rot_from_quat(geo + (size_t)qi * 5, rot);
	} else {
		rot[0] = geo[2 * (size_t)qi];
		rot[1] = geo[2 * (size_t)qi + 1];
	}
}

// W of one pixel under orientation parameters rot (see geo_setup; for RZ the
// five values of locate_rz).
template <int GEO, typename MT>
__device__ __forceinline__ double geo_sample(const double *rot, double qx, double qy, double qz, double center,
                                             long long S, const MT *__restrict__ m, double corr) {
	if constexpr (GEO == MT_3D) {
		return interp(locate(rot, qx, qy, qz, center, S), m, S, corr);
	} else if constexpr (GEO == MT_2D) {
		return interp2(locate2d(rot, qx, qy, center, S), m, S, corr);
	} else {
		return interp2(locate_rz(rot, qx, qy, center, S), m, S, corr);
	}
}

// Compensated FP32 summation (Kahan): the represented sum is s - comp, with
// an error of order n u^2 sum|x| (u = 2^-24), i.e. far below FP32 rounding.
// Intrinsics keep the compiler from simplifying (t - s) - y.
__device__ __forceinline__ void kahan_add(float &s, float &comp, float x) {
	const float y = __fsub_rn(x, comp);
	const float t = __fadd_rn(s, y);
	comp = __fsub_rn(__fsub_rn(t, s), y);
	s = t;
}

// Adds count * v exactly: the product's rounding error (from an FMA) goes
// into the compensation. The count is converted through the bits of
// 2^23 + c, without a conversion instruction.
__device__ __forceinline__ void kahan_add_count(float &s, float &comp, uint32_t count, float v) {
	const float c = __fsub_rn(__int_as_float(0x4B000000u | count), 8388608.f);
	const float p = __fmul_rn(c, v);
	const float e = __fmaf_rn(c, v, -p);
	kahan_add(s, comp, p);
	comp = __fsub_rn(comp, e);
}

// The compensated sum in FP64; -inf (a photon on a zero slice value) and NaN
// pass through (the compensation is NaN then).
__device__ __forceinline__ double kahan_value(float s, float comp) {
	return isinf(s) ? (double)s : (double)s - (double)comp;
}

// Pairs of FP32 values in one 64-bit register, for the paired FP32
// instructions of sm_100 (add/sub/fma/mul.f32x2, round to nearest per
// component): a compensated addition of two orientations costs four
// instructions instead of eight, with results identical to the scalar form.
typedef unsigned long long f32x2;
constexpr int NPAIR = LW / 2 > 0 ? LW / 2 : 1;  // pairs per lane

__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
	f32x2 d;
	asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
	return d;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
	f32x2 d;
	asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
	return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
	f32x2 d;
	asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
	return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
	f32x2 d;
	asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
	return d;
}
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
	f32x2 d;
	asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
	return d;
}
__device__ __forceinline__ void f2_unpack(f32x2 a, float &lo, float &hi) {
	asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a));
}

__device__ __forceinline__ void kahan_add2(f32x2 &s, f32x2 &comp, f32x2 x) {
	const f32x2 y = f2_sub(x, comp);
	const f32x2 t = f2_add(s, y);
	comp = f2_sub(f2_sub(t, s), y);
	s = t;
}

// count * v added exactly, as kahan_add_count, for a pair of orientations
__device__ __forceinline__ void kahan_add_count2(f32x2 &s, f32x2 &comp, uint32_t count, f32x2 v) {
	const float c = __fsub_rn(__int_as_float(0x4B000000u | count), 8388608.f);
	const f32x2 cc = f2_pack(c, c);
	const f32x2 p = f2_mul(cc, v);
	const f32x2 e = f2_fma(cc, v, p ^ 0x8000000080000000ull);  // c v - p
	kahan_add2(s, comp, p);
	comp = f2_sub(comp, e);
}

// LW consecutive floats of one lane as LW / 2 pairs (16- or 8-byte load)
__device__ __forceinline__ void ld_pairs(const float *__restrict__ p, f32x2 (&v)[NPAIR]) {
	if constexpr (LW == 4) {
		const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2 *>(p));
		v[0] = x.x;
		v[1] = x.y;
	} else {
		v[0] = __ldg(reinterpret_cast<const unsigned long long *>(p));
	}
}

// LW consecutive values of one lane as a single vector access (p aligned to
// LW elements). Read-only loads go through the non-coherent path.
__device__ __forceinline__ void ld_row(const float *__restrict__ p, float (&v)[LW]) {
	if constexpr (LW == 4) {
		const float4 x = __ldg(reinterpret_cast<const float4 *>(p));
		v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
	} else if constexpr (LW == 2) {
		const float2 x = __ldg(reinterpret_cast<const float2 *>(p));
		v[0] = x.x; v[1] = x.y;
	} else {
		v[0] = __ldg(p);
	}
}

// Same, for rows the calling kernel may have written (plain loads).
__device__ __forceinline__ void ld_row_rw(const float *p, float (&v)[LW]) {
	if constexpr (LW == 4) {
		const float4 x = *reinterpret_cast<const float4 *>(p);
		v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
	} else if constexpr (LW == 2) {
		const float2 x = *reinterpret_cast<const float2 *>(p);
		v[0] = x.x; v[1] = x.y;
	} else {
		v[0] = *p;
	}
}

__device__ __forceinline__ void st_row(float *p, const float (&v)[LW]) {
	if constexpr (LW == 4)
		*reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
	else if constexpr (LW == 2)
		*reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
	else
		*p = v[0];
}

__device__ __forceinline__ void ld_row(const double *__restrict__ p, double (&v)[LW]) {
	if constexpr (LW == 1) {
		v[0] = __ldg(p);
	} else {
#pragma unroll
		for (int k = 0; k < LW; k += 2) {
			const double2 x = __ldg(reinterpret_cast<const double2 *>(p + k));
			v[k] = x.x;
			v[k + 1] = x.y;
		}
	}
}

__device__ __forceinline__ void st_row(double *p, const double (&v)[LW]) {
	if constexpr (LW == 1) {
		*p = v[0];
	} else {
#pragma unroll
		for (int k = 0; k < LW; k += 2)
			*reinterpret_cast<double2 *>(p + k) = make_double2(v[k], v[k + 1]);
	}
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_xor_sync(FULL, v, o);
	return v;
}

}  // namespace dfg
