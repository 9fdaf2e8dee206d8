/*
 * Device helpers shared by the engine's kernels (included by .cu files only):
 * complex arithmetic, the shared-tile swizzle, the register-level gate
 * application of a pass, block reductions and cp.async wrappers.
 */
#ifndef DK_DEVICE_CUH_
#define DK_DEVICE_CUH_

#include <cuda_runtime.h>
#include <stdint.h>

#include "dk_internal.h"

namespace dk {
namespace {

template <typename R> struct CT;
template <> struct CT<double> {
	typedef double2 T;
};
template <> struct CT<float> {
	typedef float2 T;
};

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

template <typename C2> __device__ __forceinline__ C2 ldm(const double2 *p);
template <> __device__ __forceinline__ double2 ldm<double2>(const double2 *p) { return __ldg(p); }
template <> __device__ __forceinline__ float2 ldm<float2>(const double2 *p)
{
	double2 v = __ldg(p);
	return make_float2((float)v.x, (float)v.y);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
	return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
/* a * b + c */
__device__ __forceinline__ double2 cmad(double2 a, double2 b, double2 c)
{
	return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)),
			    fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cmad(float2 a, float2 b, float2 c)
{
	return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)),
			   fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ double sqabs(double2 a) { return fma(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ double sqabs(float2 a)
{
	double x = a.x, y = a.y;
	return fma(x, x, y * y);
}
__device__ __forceinline__ double2 to_c128(double2 a) { return a; }
__device__ __forceinline__ double2 to_c128(float2 a) { return make_double2(a.x, a.y); }
template <typename C2> __device__ __forceinline__ C2 from_c128(double2 a);
template <> __device__ __forceinline__ double2 from_c128<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_c128<float2>(double2 a)
{
	return make_float2((float)a.x, (float)a.y);
}

/* XOR swizzle of the shared tile: the low SW bits of the slot are XORed with
 * every higher SW-bit group, so any SW thread bits mapped to tile bits of
 * distinct residues mod SW hit distinct 16-byte (8-byte) bank groups. */
template <int SW> __device__ __forceinline__ uint32_t swz(uint32_t i)
{
	uint32_t f = 0;
#pragma unroll
	for (int s = SW; s < 20; s += SW)
		f ^= i >> s;
	return i ^ (f & ((1u << SW) - 1u));
}

/* The tile layout of a sweep header's bank map (dk_sweep_hdr.bankv): index
 * i sits in slot i ^ (XOR of nibble b of bankv over the set bits b of i). */
__device__ __forceinline__ uint32_t swz_map(uint32_t i, uint64_t bankv)
{
	uint32_t f = 0;
#pragma unroll
	for (int b = 0; b < 16; ++b)
		if ((i >> b) & 1u)
			f ^= (uint32_t)(bankv >> (4 * b)) & 15u;
	return i ^ f;
}

__device__ __forceinline__ bool ctl_ok(uint32_t loc, uint32_t lc, uint32_t la)
{
	return ((loc & lc) == lc) && !(loc & la);
}

/* ---- gate application on the 8 register amplitudes of a pass ------------
 * A pass gathers, per thread, the NA = 2^PB amplitudes that differ only in the
 * pass's PB tile bits: a[r] holds the one whose pass bits equal r, and
 * loc(r) = gb | (pass bits of r) is its tile index, needed only to evaluate
 * controls that lie inside the tile.  Template T / T0, T1 give the register
 * bit that carries gate bit 0 / 1, so every register index is a compile-time
 * constant and the amplitudes never leave registers. */
constexpr int PB = DK_PASS_BITS;
constexpr int NA = 1 << PB;

static_assert(DK_PASS_BITS == 3, "register tile of 8 amplitudes");

struct PassCtx {
	uint32_t gb, p0, p1, p2; /* raw tile index of the thread part / pass bits */
};

__device__ __forceinline__ uint32_t loc_of(const PassCtx &c, int r)
{
	return c.gb | ((r & 1) ? c.p0 : 0u) | ((r & 2) ? c.p1 : 0u) | ((r & 4) ? c.p2 : 0u);
}

template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_dense1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					 uint32_t la, const C2 *mt)
{
	const C2 m00 = mt[0], m01 = mt[1], m10 = mt[2], m11 = mt[3];
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		if (r & (1 << T))
			continue;
		const int r1 = r | (1 << T);
		if (!CTL || ctl_ok(loc_of(pc, r), lc, la)) {
			const C2 x = a[r], y = a[r1];
			a[r] = cmad(m01, y, cmul(m00, x));
			a[r1] = cmad(m11, y, cmul(m10, x));
		}
	}
}

/* [[0,1],[1,0]] (X and its controlled forms): a pure exchange */
template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_swap1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					uint32_t la)
{
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		if (r & (1 << T))
			continue;
		const int r1 = r | (1 << T);
		if (!CTL || ctl_ok(loc_of(pc, r), lc, la)) {
			const C2 x = a[r];
			a[r] = a[r1];
			a[r1] = x;
		}
	}
}

template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_anti1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					uint32_t la, const C2 *mt)
{
	const C2 m01 = mt[0], m10 = mt[1];
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		if (r & (1 << T))
			continue;
		const int r1 = r | (1 << T);
		if (!CTL || ctl_ok(loc_of(pc, r), lc, la)) {
			const C2 x = a[r], y = a[r1];
			a[r] = cmul(m01, y);
			a[r1] = cmul(m10, x);
		}
	}
}

/* diag(1, d) (Z, S, T, phase and their controlled forms): scale |1> only */
template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_phase1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					 uint32_t la, const C2 *mt)
{
	const C2 d1 = mt[0];
#pragma unroll
	for (int r = 0; r < NA; ++r)
		if ((r & (1 << T)) && (!CTL || ctl_ok(loc_of(pc, r), lc, la)))
			a[r] = cmul(d1, a[r]);
}

/* diag(1, -1) (Z, CZ and controlled forms): negate |1> only */
template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_neg1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
				       uint32_t la)
{
#pragma unroll
	for (int r = 0; r < NA; ++r)
		if ((r & (1 << T)) && (!CTL || ctl_ok(loc_of(pc, r), lc, la)))
			a[r] = mk(-a[r].x, -a[r].y);
}

template <int T, bool CTL, typename C2>
__device__ __forceinline__ void g_diag1(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					uint32_t la, const C2 *mt)
{
	const C2 d0 = mt[0], d1 = mt[1];
#pragma unroll
	for (int r = 0; r < NA; ++r)
		if (!CTL || ctl_ok(loc_of(pc, r), lc, la))
			a[r] = cmul((r & (1 << T)) ? d1 : d0, a[r]);
}

/* diagonal gate on 2 or 3 targets (runtime register bits) */
template <typename C2>
__device__ __forceinline__ void g_diagk(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					uint32_t la, int k, int t0, int t1, int t2,
					const C2 *mt)
{
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		int gi = ((r >> t0) & 1) | (((r >> t1) & 1) << 1);
		if (k > 2)
			gi |= ((r >> t2) & 1) << 2;
		if (ctl_ok(loc_of(pc, r), lc, la))
			a[r] = cmul(mt[gi], a[r]);
	}
}

template <int T0, int T1, typename C2>
__device__ __forceinline__ void g_dense2(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					 uint32_t la, const C2 *mt)
{
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		if (r & ((1 << T0) | (1 << T1)))
			continue;
		const int i1 = r | (1 << T0), i2 = r | (1 << T1), i3 = i1 | (1 << T1);
		if (!ctl_ok(loc_of(pc, r), lc, la))
			continue;
		const C2 x0 = a[r], x1 = a[i1], x2 = a[i2], x3 = a[i3];
		C2 y[4];
#pragma unroll
		for (int row = 0; row < 4; ++row) {
			C2 s = cmul(mt[4 * row], x0);
			s = cmad(mt[4 * row + 1], x1, s);
			s = cmad(mt[4 * row + 2], x2, s);
			y[row] = cmad(mt[4 * row + 3], x3, s);
		}
		a[r] = y[0];
		a[i1] = y[1];
		a[i2] = y[2];
		a[i3] = y[3];
	}
}

/* 8x8 matrix on all three register bits: a folded run of gates or a
 * 3-qubit gate.  Controls, when present, lie outside the pass bits, so they
 * hold or fail for all 8 amplitudes of the thread at once. */
template <bool CTL, typename C2>
__device__ __forceinline__ void g_dense3(C2 (&a)[NA], const PassCtx &pc, uint32_t lc,
					 uint32_t la, const C2 *mt)
{
	if (CTL && !ctl_ok(pc.gb, lc, la))
		return;
	C2 y[NA];
#pragma unroll
	for (int r = 0; r < NA; ++r) {
		C2 s = cmul(mt[NA * r], a[0]);
#pragma unroll
		for (int c = 1; c < NA; ++c)
			s = cmad(mt[NA * r + c], a[c], s);
		y[r] = s;
	}
#pragma unroll
	for (int r = 0; r < NA; ++r)
		a[r] = y[r];
}

/* One gate of a pass: a single jump on the host-computed entry code. */
template <typename C2>
__device__ __forceinline__ void apply_gate(C2 (&a)[NA], const PassCtx &pc, uint32_t code,
					   uint32_t info, uint32_t lc, uint32_t la,
					   const C2 *mt)
{
	switch (code) {
	case DK_GC_DENSE1 + 0: g_dense1<0, false>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE1 + 1: g_dense1<1, false>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE1 + 2: g_dense1<2, false>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE1 + 3: g_dense1<0, true>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE1 + 4: g_dense1<1, true>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE1 + 5: g_dense1<2, true>(a, pc, lc, la, mt); break;
	case DK_GC_SWAP1 + 0: g_swap1<0, false>(a, pc, lc, la); break;
	case DK_GC_SWAP1 + 1: g_swap1<1, false>(a, pc, lc, la); break;
	case DK_GC_SWAP1 + 2: g_swap1<2, false>(a, pc, lc, la); break;
	case DK_GC_SWAP1 + 3: g_swap1<0, true>(a, pc, lc, la); break;
	case DK_GC_SWAP1 + 4: g_swap1<1, true>(a, pc, lc, la); break;
	case DK_GC_SWAP1 + 5: g_swap1<2, true>(a, pc, lc, la); break;
	case DK_GC_PHASE1 + 0: g_phase1<0, false>(a, pc, lc, la, mt); break;
	case DK_GC_PHASE1 + 1: g_phase1<1, false>(a, pc, lc, la, mt); break;
	case DK_GC_PHASE1 + 2: g_phase1<2, false>(a, pc, lc, la, mt); break;
	case DK_GC_PHASE1 + 3: g_phase1<0, true>(a, pc, lc, la, mt); break;
	case DK_GC_PHASE1 + 4: g_phase1<1, true>(a, pc, lc, la, mt); break;
	case DK_GC_PHASE1 + 5: g_phase1<2, true>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 0: g_diag1<0, false>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 1: g_diag1<1, false>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 2: g_diag1<2, false>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 3: g_diag1<0, true>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 4: g_diag1<1, true>(a, pc, lc, la, mt); break;
	case DK_GC_DIAG1 + 5: g_diag1<2, true>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 0: g_anti1<0, false>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 1: g_anti1<1, false>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 2: g_anti1<2, false>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 3: g_anti1<0, true>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 4: g_anti1<1, true>(a, pc, lc, la, mt); break;
	case DK_GC_ANTI1 + 5: g_anti1<2, true>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 0: g_dense2<0, 1>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 1: g_dense2<0, 2>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 2: g_dense2<1, 0>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 3: g_dense2<1, 2>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 4: g_dense2<2, 0>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE2 + 5: g_dense2<2, 1>(a, pc, lc, la, mt); break;
	case DK_GC_NEG1 + 0: g_neg1<0, false>(a, pc, lc, la); break;
	case DK_GC_NEG1 + 1: g_neg1<1, false>(a, pc, lc, la); break;
	case DK_GC_NEG1 + 2: g_neg1<2, false>(a, pc, lc, la); break;
	case DK_GC_NEG1 + 3: g_neg1<0, true>(a, pc, lc, la); break;
	case DK_GC_NEG1 + 4: g_neg1<1, true>(a, pc, lc, la); break;
	case DK_GC_NEG1 + 5: g_neg1<2, true>(a, pc, lc, la); break;
	case DK_GC_DENSE3 + 0: g_dense3<false>(a, pc, lc, la, mt); break;
	case DK_GC_DENSE3 + 1: g_dense3<true>(a, pc, lc, la, mt); break;
	default:
		g_diagk(a, pc, lc, la, (info >> 6) & 3, info & 3, (info >> 2) & 3,
			(info >> 4) & 3, mt);
		break;
	}
}

/* block-wide sum of two doubles; result valid in thread 0 */
__device__ __forceinline__ void block_sum2(double &x, double &y)
{
	__shared__ double red[2][32];
	if (blockDim.x < 32) {
		/* partial warp (sweeps of registers below 8 qubits): no shuffles */
		red[0][threadIdx.x] = x;
		red[1][threadIdx.x] = y;
		__syncthreads();
		if (threadIdx.x == 0) {
			x = 0.0;
			y = 0.0;
			for (unsigned i = 0; i < blockDim.x; ++i) {
				x += red[0][i];
				y += red[1][i];
			}
		}
		__syncthreads();
		return;
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		x += __shfl_xor_sync(0xffffffffu, x, o);
		y += __shfl_xor_sync(0xffffffffu, y, o);
	}
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
	if (l == 0) {
		red[0][w] = x;
		red[1][w] = y;
	}
	__syncthreads();
	const int nw = (blockDim.x + 31) >> 5;
	if (w == 0) {
		x = l < nw ? red[0][l] : 0.0;
		y = l < nw ? red[1][l] : 0.0;
#pragma unroll
		for (int o = 16; o > 0; o >>= 1) {
			x += __shfl_xor_sync(0xffffffffu, x, o);
			y += __shfl_xor_sync(0xffffffffu, y, o);
		}
	}
	__syncthreads();
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
	const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
	const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

} // namespace
} // namespace dk

#endif
