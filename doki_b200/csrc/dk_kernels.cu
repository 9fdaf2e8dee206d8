/*
 * CUDA kernels of the B200 state-vector engine (sm_100a).
 *
 * Amplitudes are complex128 (double2) or complex64 (float2), 16 / 8 bytes,
 * qubit q = bit q of the index.  Every reduction is FP64 and deterministic:
 * blocks write partial sums into a scratch array and a single-block
 * finalize kernel adds them in a fixed order.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "dk_device.cuh"
#include "dk_kernels.h"

namespace dk {
namespace {

/* Debug builds (-DDK_DEBUG_CHECKS, libdokigpu_dbg.so): the table-driven
 * kernels check every global and shared-memory index they compute.  A failed
 * check records its site (bits 56-63) and index (bits 0-55) in g_dk_check --
 * the first failure wins -- and the access is skipped; nothing traps, so the
 * context stays usable and dk_debug_checks() reads the record.  Release
 * builds compile the checks away. */
#ifdef DK_DEBUG_CHECKS
__device__ unsigned long long g_dk_check;
__device__ __forceinline__ bool dk_in_bounds(uint64_t i, uint64_t lim, unsigned site)
{
	if (i < lim)
		return true;
	atomicCAS(&g_dk_check, 0ull,
		  ((unsigned long long)site << 56) | (i & ((1ull << 56) - 1ull)));
	return false;
}
#define DK_IN_BOUNDS(i, lim, site) dk_in_bounds((uint64_t)(i), (uint64_t)(lim), (site))
#else
#define DK_IN_BOUNDS(i, lim, site) true
#endif
enum {
	CHK_LOAD_SMEM = 1, /* tile slot of a global -> shared copy */
	CHK_LOAD_GLOBAL = 2, /* amplitude index read from the register */
	CHK_GATHER = 3, /* tile slot read by a pass */
	CHK_SCATTER = 4, /* tile slot written by a pass */
	CHK_READOUT = 5, /* tile slot read for the write-back */
	CHK_STORE = 6, /* amplitude index written to the register */
	CHK_COLLAPSE = 7, /* amplitude index read by a collapse */
	CHK_JOINT = 8 /* amplitude index read by a joint-distribution pass */
};

/* ---- fused sweep ------------------------------------------------------- */


/* Tiles of 2^m amplitudes (index bits = the sweep's qubit set, lowest
 * qubits first so a tile is made of contiguous runs) stream through shared
 * memory: cp.async brings a tile in, each pass gathers 8 amplitudes per thread
 * into registers, applies the pass's gates and scatters them back, and the
 * read-out streams the tile to `out`.  NBUF = 2: the next tile is copied into
 * the second buffer while this one is processed (one CTA per SM); NBUF = 1:
 * the next copy starts as soon as the read-out frees the buffer, overlapping
 * the global stores (two CTAs per SM).  Sums of |amp|^2 read (touched tiles)
 * and written go to per-block partials for the renormalisation. */
template <typename R, int SW, int M, int MINB, int NBUF>
__global__ void __launch_bounds__(1 << (M - DK_PASS_BITS), MINB)
	k_sweep(const typename CT<R>::T *__restrict__ in, typename CT<R>::T *out,
		const unsigned char *__restrict__ prog, double *partials)
{
	typedef typename CT<R>::T C2;
	extern __shared__ __align__(16) unsigned char sm[];
	const dk_sweep_hdr *h = reinterpret_cast<const dk_sweep_hdr *>(prog);
	const int m = h->m;
	const int lanes = m - PB;
	const uint32_t tid = threadIdx.x;
	const int npass = h->npass, ngate = h->ngate;
	const int nmat = (int)((h->bytes - h->mat_off) / 16);
	const uint32_t tn_amp = 1u << m;
	const int ncond = (int)h->ncond;
	const size_t gate_bytes = (size_t)ngate * sizeof(dk_gate_desc);
	const size_t cond_bytes = (size_t)ncond * sizeof(dk_gate_cond);
	C2 *bufs = reinterpret_cast<C2 *>(sm);
	uint4 *sg = reinterpret_cast<uint4 *>(sm + NBUF * sizeof(C2) * tn_amp);
	dk_gate_cond *scond =
		reinterpret_cast<dk_gate_cond *>(reinterpret_cast<unsigned char *>(sg) + gate_bytes);
	C2 *smat = reinterpret_cast<C2 *>(reinterpret_cast<unsigned char *>(scond) + cond_bytes);
	const dk_pass_desc *passes = reinterpret_cast<const dk_pass_desc *>(prog + h->pass_off);
	__shared__ uint8_t sq[16];
	__shared__ uint64_t soff[NA]; /* global offset of register bits (load / store) */
	__shared__ uint32_t sro[NA]; /* swizzled slot offset of the same */
	/* tile base index = OR over nibbles k of sdep[k][nibble k of the tile
	 * number]: the tile number's bits deposited into the non-tile qubits */
	__shared__ uint64_t sdep[DK_DEP_NIBBLES][16];

	{ /* stage gates and matrices (in amplitude precision) */
		const uint4 *src = reinterpret_cast<const uint4 *>(prog + h->gate_off);
		for (int i = tid; i < ngate; i += blockDim.x)
			sg[i] = __ldg(src + i);
		const uint4 *csrc = reinterpret_cast<const uint4 *>(prog + h->cond_off);
		uint4 *cdst = reinterpret_cast<uint4 *>(scond);
		for (int i = tid; i < ncond; i += blockDim.x)
			cdst[i] = __ldg(csrc + i);
		const double2 *msrc = reinterpret_cast<const double2 *>(prog + h->mat_off);
		for (int i = tid; i < nmat; i += blockDim.x)
			smat[i] = from_c128<C2>(__ldg(msrc + i));
		/* blocks can be narrower than 16 threads (registers below 7 qubits) */
		for (int i = tid; i < 16; i += blockDim.x)
			sq[i] = h->qpos[i];
	}
	__syncthreads();
	for (int r = tid; r < NA; r += blockDim.x) {
		uint64_t o = 0;
		for (int j = 0; j < PB; ++j)
			if ((r >> j) & 1)
				o |= 1ull << sq[lanes + j];
		soff[r] = o;
		sro[r] = swz<SW>((uint32_t)r << lanes);
	}
	for (int e = tid; e < DK_DEP_NIBBLES * 16; e += blockDim.x) {
		uint64_t v = (uint64_t)(e & 15) << (4 * (e >> 4));
		for (int j = 0; j < m; ++j) {
			const int q = sq[j];
			v = ((v >> q) << (q + 1)) | (v & ((1ull << q) - 1ull));
		}
		sdep[e >> 4][e & 15] = v;
	}
	uint64_t off_t = 0;
	for (int j = 0; j < lanes; ++j)
		if ((tid >> j) & 1u)
			off_t |= 1ull << sq[j];
	const uint32_t stid = swz<SW>(tid);
	__syncthreads();
	const uint64_t ntiles = h->ntiles;
	const int ndep = (h->n - m + 3) >> 2;
	const bool skip_idle = (in == out) && !h->all_touched;

	auto tile_base = [&](uint64_t t) -> uint64_t {
		uint64_t base = 0;
#pragma unroll
		for (int k = 0; k < DK_DEP_NIBBLES; ++k)
			if (k < ndep)
				base |= sdep[k][(t >> (4 * k)) & 15u];
		return base;
	};
	/* next tile (>= t, stepping by the grid) with at least one active gate */
	auto next_tile = [&](uint64_t t) -> uint64_t {
		for (; t < ntiles; t += gridDim.x) {
			if (!skip_idle)
				return t;
			const uint64_t base = tile_base(t);
			for (int g = 0; g < ngate; ++g) {
				const uint32_t gi = sg[g].y & 0xffffu;
				if (gi == 0xffffu)
					return t;
				const dk_gate_cond c = scond[gi];
				if (((base & c.gc) == c.gc) && !(base & c.ga))
					return t;
			}
		}
		return ntiles;
	};
	[[maybe_unused]] const uint64_t nglob = 1ull << h->n;
	auto prefetch = [&](uint64_t base, C2 *buf) {
		const uint64_t bo = base | off_t;
#pragma unroll
		for (int r = 0; r < NA; ++r) {
			const uint32_t so = stid ^ sro[r];
			const uint64_t gi = bo | soff[r];
			if (!DK_IN_BOUNDS(so, tn_amp, CHK_LOAD_SMEM) ||
			    !DK_IN_BOUNDS(gi, nglob, CHK_LOAD_GLOBAL))
				continue;
			C2 *dst = buf + so;
			if (sizeof(C2) == 16)
				cp_async16(dst, in + gi);
			else
				cp_async8(dst, in + gi);
		}
		cp_async_commit();
	};
	/* slot offsets of the next pass, loaded while the current one computes */
	uint32_t nsgb, ns0, ns1, ns2;
	auto pass_slots = [&](int p) {
		const dk_pass_desc *pd = passes + p;
		nsgb = __ldg(&pd->slo[tid & 31]) ^ __ldg(&pd->shi[tid >> 5]);
		ns0 = __ldg(&pd->sp[0]);
		ns1 = __ldg(&pd->sp[1]);
		ns2 = __ldg(&pd->sp[2]);
	};
	pass_slots(0);

	double insq = 0.0, outsq = 0.0;
	uint64_t t = next_tile(blockIdx.x);
	if (t < ntiles)
		prefetch(tile_base(t), bufs);
	int cur = 0;
	while (t < ntiles) {
		const uint64_t base = tile_base(t);
		C2 *tile = bufs + (NBUF == 2 ? cur * tn_amp : 0);
		uint64_t tn = ntiles;
		if (NBUF == 2) {
			tn = next_tile(t + gridDim.x);
			if (tn < ntiles) {
				prefetch(tile_base(tn), bufs + (cur ^ 1) * tn_amp);
				asm volatile("cp.async.wait_group 1;\n" ::);
			} else {
				cp_async_wait_all();
			}
		} else {
			cp_async_wait_all();
		}
		__syncthreads();
		C2 a[NA];
		for (int p = 0; p < npass; ++p) {
			const dk_pass_desc *pd = passes + p;
			const uint32_t sgb = nsgb, s0 = ns0, s1 = ns1, s2 = ns2;
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t sl = sgb ^ ((r & 1) ? s0 : 0u) ^ ((r & 2) ? s1 : 0u) ^
						    ((r & 4) ? s2 : 0u);
				a[r] = DK_IN_BOUNDS(sl, tn_amp, CHK_GATHER) ? tile[sl] : C2{};
			}
			if (p == 0) {
#pragma unroll
				for (int r = 0; r < NA; ++r)
					insq += sqabs(a[r]);
			}
			pass_slots(p + 1 < npass ? p + 1 : 0);
			const uint32_t pflags = __ldg(&pd->flags);
			PassCtx pc;
			if (pflags & DK_PASS_CTL) {
				pc.gb = __ldg(&pd->rlo[tid & 31]) | __ldg(&pd->rhi[tid >> 5]);
				pc.p0 = __ldg(&pd->pm[0]);
				pc.p1 = __ldg(&pd->pm[1]);
				pc.p2 = __ldg(&pd->pm[2]);
			} else {
				pc.gb = pc.p0 = pc.p1 = pc.p2 = 0;
			}
			const int g1 = __ldg(&pd->g1);
			for (int g = __ldg(&pd->g0); g < g1; ++g) {
				const uint4 d = sg[g];
				const uint32_t gi = d.y & 0xffffu;
				if (gi != 0xffffu) {
					const dk_gate_cond c = scond[gi];
					if (((base & c.gc) != c.gc) || (base & c.ga))
						continue;
				}
				apply_gate(a, pc, d.x & 0xffffu, d.y >> 16, d.z, d.w, smat + (d.x >> 16));
			}
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t sl = sgb ^ ((r & 1) ? s0 : 0u) ^ ((r & 2) ? s1 : 0u) ^
						    ((r & 4) ? s2 : 0u);
				if (DK_IN_BOUNDS(sl, tn_amp, CHK_SCATTER))
					tile[sl] = a[r];
			}
			/* the flag is uniform over the block */
			if (pflags & DK_PASS_WARP)
				__syncwarp();
			else
				__syncthreads();
		}
#pragma unroll
		for (int r = 0; r < NA; ++r) {
			const uint32_t so = stid ^ sro[r];
			a[r] = DK_IN_BOUNDS(so, tn_amp, CHK_READOUT) ? tile[so] : C2{};
		}
		if (NBUF == 1) {
			__syncthreads(); /* the buffer is free: start the next tile's copy */
			tn = next_tile(t + gridDim.x);
			if (tn < ntiles)
				prefetch(tile_base(tn), bufs);
		}
		const uint64_t bo = base | off_t;
#pragma unroll
		for (int r = 0; r < NA; ++r) {
			outsq += sqabs(a[r]);
			if (DK_IN_BOUNDS(bo | soff[r], nglob, CHK_STORE))
				__stcs(out + (bo | soff[r]), a[r]);
		}
		if (NBUF == 2)
			__syncthreads(); /* this buffer is refilled two tiles later */
		t = tn;
		cur ^= 1;
	}
	cp_async_wait_all();
	block_sum2(insq, outsq);
	if (tid == 0) {
		partials[2 * blockIdx.x] = insq;
		partials[2 * blockIdx.x + 1] = outsq;
	}
}

/* ---- tensor-core sweep --------------------------------------------------- */

#ifndef DK_TC_MINB11
#define DK_TC_MINB11 3
#endif
#ifndef DK_TC_MINB12
#define DK_TC_MINB12 3
#endif


/* FP64 tensor-core MMA, D (8x8) += A (8x4, row-major) * B (4x8, column-major).
 * Lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)], D[l/4][2(l%4)+1]. */
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
	asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
	    : "+d"(d0), "+d"(d1)
	    : "d"(a), "d"(b));
}

/* Sweep whose gate list holds only 8x8 matrices in register order (folded
 * runs of gates, and single gates whose remaining controls lie off the pass
 * bits or outside the tile).  A pass works on columns: the 8 amplitudes that
 * differ only in the pass bits, one column per thread index as in k_sweep.
 * A warp owns 32 columns and treats them as 4 groups of 8; each group is one
 * real product  [yr; yi] = [[Mr, -Mi], [Mi, Mr]] [xr; xi]  (16x16 by 16x8),
 * i.e. 2 row blocks x 4 k-steps of m8n8k4 FP64 MMAs.  Lane l gathers
 * amplitudes l%4 and 4 + l%4 of column l/4 (its B fragments), holds matrix
 * entries (l/4, l%4) and (l/4, 4 + l%4) (its A fragments, read through L1),
 * and writes amplitude l/4 of columns 2(l%4) and 2(l%4)+1.  Entries with
 * controls off the pass bits write only the columns whose tile index
 * satisfies them; the others keep their values in the shared tile. */
/* Matrix of a gate-list entry of a tensor sweep (whole 8x8 matrices), the
 * tile's variant picked by its conditions. */
__device__ __forceinline__ uint32_t tc_matrix(const uint4 &d, const dk_gate_cond *scond,
					      uint64_t base)
{
	uint32_t mi = d.x >> 16;
	if ((d.x & 0xffffu) == DK_GC_DENSE3V)
		for (uint32_t c = 0; c < d.w; ++c) {
			const dk_gate_cond cc = scond[(d.z >> (10 * c)) & 1023u];
			if (((base & cc.gc) == cc.gc) && !(base & cc.ga))
				mi += 1u << c;
		}
	return mi;
}

/* y = M x for one column group, Gauss form: Mr xr, Mi xi, (Mr + Mi)(xr + xi)
 * as three real 8x8 products of two k-steps each; y = (yr[2t], yr[2t+1],
 * yi[2t], yi[2t+1]) of output amplitude l/4. */
__device__ __forceinline__ void tc_product(const double2 &e0, const double2 &e1, const double2 &x0,
					   const double2 &x1, double (&y)[4])
{
	double p1[2] = { 0.0, 0.0 }, p2[2] = { 0.0, 0.0 }, p3[2] = { 0.0, 0.0 };
	dmma(p1[0], p1[1], e0.x, x0.x);
	dmma(p2[0], p2[1], e0.y, x0.y);
	dmma(p3[0], p3[1], e0.x + e0.y, x0.x + x0.y);
	dmma(p1[0], p1[1], e1.x, x1.x);
	dmma(p2[0], p2[1], e1.y, x1.y);
	dmma(p3[0], p3[1], e1.x + e1.y, x1.x + x1.y);
	y[0] = p1[0] - p2[0];
	y[1] = p1[1] - p2[1];
	y[2] = p3[0] - p1[0] - p2[0];
	y[3] = p3[1] - p1[1] - p2[1];
}

/* TF32 tensor-core MMA, D (16x8, f32) += A (16x8, row-major) * B (8x8,
 * column-major).  Lane l = 4 g + t holds A[g][t], A[g+8][t], A[g][t+4],
 * A[g+8][t+4], B[t][g], B[t+4][g] and D[g][2t], D[g][2t+1], D[g+8][2t],
 * D[g+8][2t+1]: the B and D lane layouts of the FP64 m8n8k4 MMA above. */
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
					 uint32_t b1)
{
	asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
	    "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
	    : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
	    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

/* x = hi + lo exactly, hi = x with its 13 low mantissa bits cleared (a TF32
 * value).  The MMA reads lo as TF32 too (its low 13 bits ignored), so hi + lo
 * reaches the product with about 21 bits of x. */
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo)
{
	hi = __float_as_uint(x) & 0xffffe000u;
	lo = __float_as_uint(x - __uint_as_float(hi));
}

/* Lane fragments of one 8x8 matrix entry and the column-group product y = M x
 * of a tensor sweep, per amplitude precision.  complex128: FP64 MMAs in the
 * Gauss form (tc_product).  complex64: the real form
 *   [yr; yi] = [[Mr, -Mi], [Mi, Mr]] [xr; xi]
 * as one 16x16-by-16x8 product, i.e. two k-steps of the TF32 m16n8k8 MMA
 * (k-step 0 multiplies xr by [Mr; Mi], k-step 1 xi by [-Mi; Mr]).  Operands
 * are split into TF32 hi + lo parts and each k-step takes hi*hi + hi*lo +
 * lo*hi (the lo*lo term is below FP32 rounding), accumulated in FP32, so the
 * product carries close to FP32 precision.  Lane l = 4 g + t reads matrix entries
 * (g, t) and (g, t + 4) in both precisions. */
template <typename R> struct TcFrag;

template <> struct TcFrag<double> {
	double2 e0, e1;
	__device__ __forceinline__ void load(const double2 *mt)
	{
		e0 = __ldg(mt);
		e1 = __ldg(mt + 4);
	}
	__device__ __forceinline__ void product(const double2 &x0, const double2 &x1,
						double (&y)[4]) const
	{
		tc_product(e0, e1, x0, x1, y);
	}
};

template <> struct TcFrag<float> {
	uint32_t k0h[4], k0l[4], k1h[4], k1l[4];
	__device__ __forceinline__ void load(const double2 *mt)
	{
		const double2 e0 = __ldg(mt), e1 = __ldg(mt + 4);
		const float a0[4] = { (float)e0.x, (float)e0.y, (float)e1.x, (float)e1.y };
		const float a1[4] = { -(float)e0.y, (float)e0.x, -(float)e1.y, (float)e1.x };
#pragma unroll
		for (int i = 0; i < 4; ++i) {
			tf32_split(a0[i], k0h[i], k0l[i]);
			tf32_split(a1[i], k1h[i], k1l[i]);
		}
	}
	__device__ __forceinline__ void product(const float2 &x0, const float2 &x1,
						float (&y)[4]) const
	{
		uint32_t r0h, r0l, r1h, r1l, i0h, i0l, i1h, i1l;
		tf32_split(x0.x, r0h, r0l);
		tf32_split(x1.x, r1h, r1l);
		tf32_split(x0.y, i0h, i0l);
		tf32_split(x1.y, i1h, i1l);
		/* one accumulation chain over both k-steps, small terms first
		 * (no final add of two partial sums) */
		y[0] = y[1] = y[2] = y[3] = 0.0f;
		mma_tf32(y, k0l, r0h, r1h);
		mma_tf32(y, k1l, i0h, i1h);
		mma_tf32(y, k0h, r0l, r1l);
		mma_tf32(y, k1h, i0l, i1l);
		mma_tf32(y, k0h, r0h, r1h);
		mma_tf32(y, k1h, i0h, i1h);
	}
};

template <typename C2, typename R> __device__ __forceinline__ C2 c2_make(R re, R im);
template <> __device__ __forceinline__ double2 c2_make<double2, double>(double re, double im)
{
	return make_double2(re, im);
}
template <> __device__ __forceinline__ float2 c2_make<float2, float>(float re, float im)
{
	return make_float2(re, im);
}

template <typename R, int SW, int M, int MINB>
__global__ void __launch_bounds__(1 << ((M < 11 ? M : 11) - DK_PASS_BITS), MINB)
	k_sweep_tc(const typename CT<R>::T *__restrict__ in, typename CT<R>::T *out,
		   const unsigned char *__restrict__ prog, double *partials)
{
	typedef typename CT<R>::T C2;
	extern __shared__ __align__(16) unsigned char sm[];
	const dk_sweep_hdr *h = reinterpret_cast<const dk_sweep_hdr *>(prog);
	const int m = h->m;
	const int lanes = m - PB;
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	/* 12-bit tiles: 256 threads, thread t owns columns t and t + 256 */
	constexpr int VT = (M >= 12) ? 2 : 1;
	const int npass = h->npass, ngate = h->ngate;
	const uint32_t tn_amp = 1u << m;
	const int ncond = (int)h->ncond;
	const size_t gate_bytes = (size_t)ngate * sizeof(dk_gate_desc);
	C2 *const bufs = reinterpret_cast<C2 *>(sm);
	uint4 *sg = reinterpret_cast<uint4 *>(sm + sizeof(C2) * tn_amp);
	dk_gate_cond *scond =
		reinterpret_cast<dk_gate_cond *>(reinterpret_cast<unsigned char *>(sg) + gate_bytes);
	const dk_pass_desc *passes = reinterpret_cast<const dk_pass_desc *>(prog + h->pass_off);
	const double2 *mats = reinterpret_cast<const double2 *>(prog + h->mat_off);
	__shared__ uint8_t sq[16];
	__shared__ uint64_t soff[NA];
	__shared__ uint32_t sro[NA];
	__shared__ uint64_t sdep[DK_DEP_NIBBLES][16];

	{
		const uint4 *src = reinterpret_cast<const uint4 *>(prog + h->gate_off);
		for (int i = tid; i < ngate; i += blockDim.x)
			sg[i] = __ldg(src + i);
		const uint4 *csrc = reinterpret_cast<const uint4 *>(prog + h->cond_off);
		uint4 *cdst = reinterpret_cast<uint4 *>(scond);
		for (int i = tid; i < ncond; i += blockDim.x)
			cdst[i] = __ldg(csrc + i);
		for (int i = tid; i < 16; i += blockDim.x)
			sq[i] = h->qpos[i];
	}
	__syncthreads();
	for (int r = tid; r < NA; r += blockDim.x) {
		uint64_t o = 0;
		for (int j = 0; j < PB; ++j)
			if ((r >> j) & 1)
				o |= 1ull << sq[lanes + j];
		soff[r] = o;
		sro[r] = swz_map((uint32_t)r << lanes, h->bankv);
	}
	for (int e = tid; e < DK_DEP_NIBBLES * 16; e += blockDim.x) {
		uint64_t v = (uint64_t)(e & 15) << (4 * (e >> 4));
		for (int j = 0; j < m; ++j) {
			const int q = sq[j];
			v = ((v >> q) << (q + 1)) | (v & ((1ull << q) - 1ull));
		}
		sdep[e >> 4][e & 15] = v;
	}
	/* column set h of this thread: thread index tid + 256 h; the second set
	 * differs in thread bit 8 only, so its offsets follow from the first */
	uint64_t off_t0 = 0;
	for (int j = 0; j < lanes; ++j)
		if ((tid >> j) & 1u)
			off_t0 |= 1ull << sq[j];
	const uint32_t stid0 = swz_map(tid, h->bankv);
	const uint32_t s256 = swz_map(256u, h->bankv);
	auto off_t = [&](int h) -> uint64_t { return h ? (off_t0 | (1ull << sq[8])) : off_t0; };
	auto stid = [&](int h) -> uint32_t { return h ? (stid0 ^ s256) : stid0; };
	__syncthreads();
	const uint64_t ntiles = h->ntiles;
	const int ndep = (h->n - m + 3) >> 2;
	const bool skip_idle = (in == out) && !h->all_touched;

	auto tile_base = [&](uint64_t t) -> uint64_t {
		uint64_t base = 0;
#pragma unroll
		for (int k = 0; k < DK_DEP_NIBBLES; ++k)
			if (k < ndep)
				base |= sdep[k][(t >> (4 * k)) & 15u];
		return base;
	};
	auto next_tile = [&](uint64_t t) -> uint64_t {
		for (; t < ntiles; t += gridDim.x) {
			if (!skip_idle)
				return t;
			const uint64_t base = tile_base(t);
			for (int g = 0; g < ngate; ++g) {
				const uint32_t gi = sg[g].y & 0xffffu;
				if (gi == 0xffffu)
					return t;
				const dk_gate_cond c = scond[gi];
				if (((base & c.gc) == c.gc) && !(base & c.ga))
					return t;
			}
		}
		return ntiles;
	};
	[[maybe_unused]] const uint64_t nglob = 1ull << h->n;
	auto prefetch = [&](uint64_t base, C2 *buf) {
#pragma unroll
		for (int h = 0; h < VT; ++h) {
			const uint64_t bo = base | off_t(h);
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t so = stid(h) ^ sro[r];
				const uint64_t gi = bo | soff[r];
				if (!DK_IN_BOUNDS(so, tn_amp, CHK_LOAD_SMEM) ||
				    !DK_IN_BOUNDS(gi, nglob, CHK_LOAD_GLOBAL))
					continue;
				C2 *dst = buf + so;
				if (sizeof(C2) == 16)
					cp_async16(dst, in + gi);
				else
					cp_async8(dst, in + gi);
			}
		}
		cp_async_commit();
	};

	double insq = 0.0, outsq = 0.0;
	uint64_t t = next_tile(blockIdx.x);
	if (t < ntiles)
		prefetch(tile_base(t), bufs);
	const uint32_t gl = lane >> 2, gk = lane & 3u;
	while (t < ntiles) {
		const uint64_t base = tile_base(t);
		C2 *const tile = bufs;
		uint64_t tn = ntiles;
		cp_async_wait_all();
		__syncthreads();
		if (skip_idle) {
			/* only touched tiles reach here: their old |amp|^2 leaves csq.
			 * The read uses the identity mapping, so every thread must be
			 * done with it before the first pass writes the tile. */
#pragma unroll
			for (int h = 0; h < VT; ++h)
#pragma unroll
				for (int r = 0; r < NA; ++r) {
					const uint32_t so = stid(h) ^ sro[r];
					if (DK_IN_BOUNDS(so, tn_amp, CHK_READOUT))
						insq += sqabs(tile[so]);
				}
			__syncthreads();
		}
		for (int p = 0; p < npass; ++p) {
			const dk_pass_desc *pd = passes + p;
			if (__ldg(&pd->flags) & DK_PASS_CHAIN) {
				/* this pass and the next, one entry each: this pass's
				 * MMA output is the next pass's MMA input in place */
				const dk_pass_desc *pn = pd + 1;
				const uint32_t t8 = __ldg(&pd->slo[8]), t16 = __ldg(&pd->slo[16]);
				const uint32_t sgl0 = __ldg(&pd->slo[gl]);
				const uint32_t s0 = __ldg(&pd->sp[0]), s1 = __ldg(&pd->sp[1]),
					       s2 = __ldg(&pd->sp[2]);
				const uint32_t gj0 = ((gk & 1u) ? s0 : 0u) ^ ((gk & 2u) ? s1 : 0u);
				const uint32_t gj1 = gj0 ^ s2;
				const uint32_t u8 = __ldg(&pn->slo[8]), u16 = __ldg(&pn->slo[16]);
				const uint32_t sgk0 = __ldg(&pn->slo[2u * gk]), u1 = __ldg(&pn->slo[1]);
				const uint32_t n0 = __ldg(&pn->sp[0]), n1 = __ldg(&pn->sp[1]),
					       n2 = __ldg(&pn->sp[2]);
				const uint32_t sr = ((gl & 1u) ? n0 : 0u) ^ ((gl & 2u) ? n1 : 0u) ^
						    ((gl & 4u) ? n2 : 0u);
				/* lane fragments: entries (l/4, l%4) and (l/4, 4 + l%4) */
				const double2 *ma = mats + 64 * (size_t)tc_matrix(sg[__ldg(&pd->g0)],
										  scond, base) +
						    8 * gl + gk;
				const double2 *mb = mats + 64 * (size_t)tc_matrix(sg[__ldg(&pn->g0)],
										  scond, base) +
						    8 * gl + gk;
				/* the second entry's fragments are reloaded per group (L1),
				 * which keeps three CTAs per SM */
				TcFrag<R> fa, fb;
				fa.load(ma);
#pragma unroll
				for (int hq = 0; hq < 4 * VT; ++hq) {
					const int q = hq & 3, h = hq >> 2;
					const uint32_t sgl = sgl0 ^ __ldg(&pd->shi[warp + 8u * h]);
					const uint32_t sgk = sgk0 ^ __ldg(&pn->shi[warp + 8u * h]);
					const uint32_t bg = sgl ^ ((q & 1) ? t8 : 0u) ^ ((q & 2) ? t16 : 0u);
					const C2 x0 = DK_IN_BOUNDS(bg ^ gj0, tn_amp, CHK_GATHER) ? tile[bg ^ gj0]
												 : C2{};
					const C2 x1 = DK_IN_BOUNDS(bg ^ gj1, tn_amp, CHK_GATHER) ? tile[bg ^ gj1]
												 : C2{};
					R y[4], z[4];
					fa.product(x0, x1, y);
					fb.load(mb);
					/* amplitude l%4 and 4 + l%4 of column l/4 in the next pass */
					fb.product(c2_make<C2, R>(y[0], y[2]), c2_make<C2, R>(y[1], y[3]), z);
					__syncwarp(); /* the group's gathers precede its writes */
#pragma unroll
					for (int e = 0; e < 2; ++e) {
						const uint32_t bs = sgk ^ (e ? u1 : 0u) ^ ((q & 1) ? u8 : 0u) ^
								    ((q & 2) ? u16 : 0u);
						if (DK_IN_BOUNDS(bs ^ sr, tn_amp, CHK_SCATTER))
							tile[bs ^ sr] = c2_make<C2, R>(z[e], z[2 + e]);
					}
				}
				__syncwarp();
				++p;
				if (!(__ldg(&pn->flags) & DK_PASS_WARP))
					__syncthreads();
				continue;
			}
			/* the slot tables are XOR-linear in the thread index: a column's
			 * slot is the XOR of the entries of its set bits */
			const uint32_t t8 = __ldg(&pd->slo[8]), t16 = __ldg(&pd->slo[16]);
			const uint32_t sgl0 = __ldg(&pd->slo[gl]);
			const uint32_t sgk0 = __ldg(&pd->slo[2u * gk]), t1 = __ldg(&pd->slo[1]);
			const uint32_t s0 = __ldg(&pd->sp[0]), s1 = __ldg(&pd->sp[1]),
				       s2 = __ldg(&pd->sp[2]);
			const uint32_t gj0 = ((gk & 1u) ? s0 : 0u) ^ ((gk & 2u) ? s1 : 0u);
			const uint32_t gj1 = gj0 ^ s2;
			const uint32_t sr = ((gl & 1u) ? s0 : 0u) ^ ((gl & 2u) ? s1 : 0u) ^
					    ((gl & 4u) ? s2 : 0u);
			const uint32_t pflags = __ldg(&pd->flags);
			const int g1 = __ldg(&pd->g1);
			for (int g = __ldg(&pd->g0); g < g1; ++g) {
				const uint4 d = sg[g];
				const uint32_t gi = d.y & 0xffffu;
				if (gi != 0xffffu) {
					const dk_gate_cond c = scond[gi];
					if (((base & c.gc) != c.gc) || (base & c.ga))
						continue;
				}
				/* lane fragments: entries (l/4, l%4) and (l/4, 4 + l%4) */
				const double2 *mt = mats + 64 * (size_t)tc_matrix(d, scond, base) + 8 * gl + gk;
				TcFrag<R> fa;
				fa.load(mt);
				const bool ctl = (d.x & 0xffffu) == DK_GC_DENSE3 + 1;
				/* one column group at a time: the groups' slots are
				 * disjoint */
#pragma unroll
				for (int hq = 0; hq < 4 * VT; ++hq) {
					const int q = hq & 3, h = hq >> 2;
					const uint32_t shw = __ldg(&pd->shi[warp + 8u * h]);
					const uint32_t sgl = sgl0 ^ shw, sgk = sgk0 ^ shw;
					const uint32_t bg = sgl ^ ((q & 1) ? t8 : 0u) ^ ((q & 2) ? t16 : 0u);
					const C2 x0 = DK_IN_BOUNDS(bg ^ gj0, tn_amp, CHK_GATHER) ? tile[bg ^ gj0]
												 : C2{};
					const C2 x1 = DK_IN_BOUNDS(bg ^ gj1, tn_amp, CHK_GATHER) ? tile[bg ^ gj1]
												 : C2{};
					R y[4];
					fa.product(x0, x1, y);
					__syncwarp(); /* the group's gathers precede its writes */
#pragma unroll
					for (int e = 0; e < 2; ++e) {
						if (ctl) { /* rare: controls off the pass bits */
							const uint32_t col = (q << 3) | (2u * gk + e);
							const uint32_t raw = __ldg(&pd->rlo[col]) |
									     __ldg(&pd->rhi[warp + 8u * h]);
							if (!ctl_ok(raw, d.z, d.w))
								continue;
						}
						const uint32_t bs = sgk ^ (e ? t1 : 0u) ^ ((q & 1) ? t8 : 0u) ^
								    ((q & 2) ? t16 : 0u);
						if (DK_IN_BOUNDS(bs ^ sr, tn_amp, CHK_SCATTER))
							tile[bs ^ sr] = c2_make<C2, R>(y[e], y[2 + e]);
					}
				}
				__syncwarp();
			}
			if (!(pflags & DK_PASS_WARP))
				__syncthreads();
		}
		if (VT == 1) {
			C2 a[NA];
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t so = stid(0) ^ sro[r];
				a[r] = DK_IN_BOUNDS(so, tn_amp, CHK_READOUT) ? tile[so] : C2{};
			}
			__syncthreads(); /* the buffer is free */
			tn = next_tile(t + gridDim.x);
			if (tn < ntiles)
				prefetch(tile_base(tn), bufs);
			const uint64_t bo = base | off_t(0);
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				outsq += sqabs(a[r]);
				if (DK_IN_BOUNDS(bo | soff[r], nglob, CHK_STORE))
					__stcs(out + (bo | soff[r]), a[r]);
			}
		} else {
			/* two column sets: stream each amplitude out as it is read */
#pragma unroll
			for (int h = 0; h < VT; ++h) {
				const uint64_t bo = base | off_t(h);
#pragma unroll
				for (int r = 0; r < NA; ++r) {
					const uint32_t so = stid(h) ^ sro[r];
					const C2 v = DK_IN_BOUNDS(so, tn_amp, CHK_READOUT) ? tile[so] : C2{};
					outsq += sqabs(v);
					if (DK_IN_BOUNDS(bo | soff[r], nglob, CHK_STORE))
						__stcs(out + (bo | soff[r]), v);
				}
			}
			__syncthreads(); /* the buffer is free */
			tn = next_tile(t + gridDim.x);
			if (tn < ntiles)
				prefetch(tile_base(tn), bufs);
		}
		t = tn;
	}
	cp_async_wait_all();
	block_sum2(insq, outsq);
	if (tid == 0) {
		partials[2 * blockIdx.x] = insq;
		partials[2 * blockIdx.x + 1] = outsq;
	}
}

/* ---- complex64 tensor sweep on tcgen05 (tensor memory) --------------------
 *
 * The same sweep programs as k_sweep_tc (12-bit tiles, every entry an 8x8
 * complex matrix in register order), with each entry applied by the 5th-gen
 * tensor cores.  The 512 columns of a tile (8 amplitudes that differ only in
 * the pass bits) are the rows of A; one entry is
 *     Y^T (512 x 16) = X^T (512 x 16) R^T,   R = [[Mr, -Mi], [Mi, Mr]],
 * x = (re0..re7, im0..im7) of a column, as 4 row blocks of M = 128 (one
 * tensor-memory lane per column), K = 16 (two k-steps of 8).  Operands are
 * split into TF32 hi + lo parts (as in the mma.sync form).  B of an entry is
 * B' = [R_hi; R_lo] (32 x 16), so one N = 32 product A_hi B'^T gives
 * hi*hi in D columns 0..15 and hi*lo in 16..31, and an N = 16 product
 * A_lo R_hi^T accumulates lo*hi into 16..31: four MMAs per row block, and
 * y = D[0..15] + D[16..31] (the small terms summed apart from hi*hi).  A
 * lives in tensor memory (written by the threads that gathered the columns,
 * tcgen05.st), B' in shared memory in the K-major layout without swizzle
 * (split once per CTA for all matrices of the sweep when they fit, else per
 * entry), D in tensor memory.  The two warpgroups work on separate halves
 * of the tile: each gathers its two row blocks, passes a 128-thread barrier,
 * has one thread issue its 8 MMAs and commit them to its own mbarrier, and
 * reads back its own rows (tcgen05.ld), so a column never leaves the thread
 * that owns it between gather and scatter, and one half's MMAs run while the
 * other half gathers or scatters.
 *
 * Tensor-memory columns per CTA (256): A hi [0, 64), A lo [64, 128) -- 16
 * per row block -- and D [128, 256), 32 per row block.  The launch keeps at
 * most two CTAs of any such kernel per SM (shared memory), so 2 x 256 <= 512
 * columns and the allocation never waits.  Warp w owns row blocks 2 (w / 4)
 * and 2 (w / 4) + 1 in lanes 32 (w % 4) .. + 31: column c = 128 b +
 * 32 (w % 4) + lane.  Every wait on the MMAs is bounded: on expiry the
 * kernel counts the fault in g_dk_tm_fault, waits (bounded) for the MMAs in
 * flight, frees its tensor memory and returns; the host reports
 * DK_ERR_TIMEOUT at the next read. */
__device__ unsigned int g_dk_tm_fault;
#ifdef DK_DEBUG_CHECKS
/* Debug builds only, a test hook: while set, the issuing threads of a
 * tcgen05 sweep issue no MMA and no commit, so every wait runs out on an
 * mbarrier that nothing arrives at (dk_debug_tm_starve). */
__device__ int g_dk_tm_starve;
#define DK_TM_STARVED() (g_dk_tm_starve != 0)
#else
#define DK_TM_STARVED() false
#endif

constexpr int kTmCols = 256; /* tensor-memory columns per CTA */
/* A wait on the MMAs gives up after this long (ns of %globaltimer); the
 * poll count is a second bound in case the timer does not advance. */
constexpr unsigned long long kTmWaitNs = 1000000000ull;
constexpr int kTmWaitPolls = 1 << 26;
/* floats of one B' operand: two k-steps of 32 rows x 8 */
constexpr int kTmBFloats = 512;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

/* Shared-memory matrix descriptor: K-major, no swizzle, core matrices of 8
 * rows x 16 bytes; LBO = 128 B between the two 16-byte K chunks of a k-step,
 * SBO = 256 B between 8-row groups; descriptor version 1. */
__device__ __forceinline__ uint64_t umma_desc_k(uint32_t addr)
{
	return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) |
	       ((uint64_t)(256u >> 4) << 32) | ((uint64_t)1 << 46);
}

/* Offset (in floats) of B'(n, k), n < 32, in a buffer of that layout:
 * k-steps of 8 at 256 floats (1 KiB), 8-row groups at 64, K chunks of 4 at
 * 32, rows at 4. */
__device__ __forceinline__ int umma_b_off(int n, int k)
{
	return (k >> 3) * 256 + (n >> 3) * 64 + ((k & 7) >> 2) * 32 + (n & 7) * 4 + (k & 3);
}

/* kind::tf32, D f32, A and B K-major, M = 128, N = 16 or 32 */
constexpr uint32_t kTmIdesc16 = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) |
				((128u >> 4) << 24);
constexpr uint32_t kTmIdesc32 = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) |
				((128u >> 4) << 24);

__device__ __forceinline__ void umma_tf32_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc,
					     uint32_t acc)
{
	const uint32_t zero = 0;
	asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
		     "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %5, %5, %5}, p;\n\t}"
		     ::"r"(d), "r"(a), "l"(b), "r"(idesc), "r"(acc), "r"(zero));
}

__device__ __forceinline__ void tm_st16(uint32_t ta, const uint32_t (&v)[16])
{
	asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, "
		     "%8, %9, %10, %11, %12, %13, %14, %15, %16};" ::"r"(ta),
		     "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
		     "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
		     "r"(v[14]), "r"(v[15]));
}

__device__ __forceinline__ void tm_ld16(uint32_t ta, uint32_t (&v)[16])
{
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
		     "%9, %10, %11, %12, %13, %14, %15}, [%16];"
		     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
		       "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
		       "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
		     : "r"(ta));
}

/* Wait for the mbarrier's phase `parity` to complete, for at most kTmWaitNs
 * (and kTmWaitPolls polls); false when the limit ran out. */
__device__ __forceinline__ bool tm_wait(uint32_t mbar, uint32_t parity)
{
	unsigned long long t0, t1;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
	for (int it = 0; it < kTmWaitPolls; ++it) {
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			     "selp.u32 %0, 1, 0, p;\n\t}"
			     : "=r"(done)
			     : "r"(mbar), "r"(parity));
		if (done)
			return true;
		asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
		if (t1 - t0 > kTmWaitNs)
			return false;
	}
	return false;
}

/* Write B' = [R_hi; R_lo] of one 8x8 complex matrix (64 complex entries in
 * register order, entry (r, c) at 8 r + c) into `b` (kTmBFloats floats),
 * element e of the 256 of R handled by the calling thread for e = e0,
 * e0 + stride, ... */
template <typename E>
__device__ __forceinline__ void tm_write_b(float *b, const E *mt, int e0, int stride)
{
	for (int e = e0; e < 256; e += stride) {
		const int n = e >> 4, k = e & 15;
		const E x = mt[8 * (n & 7) + (k & 7)];
		const float re = (float)x.x, im = (float)x.y;
		const float v = ((n < 8) == (k < 8)) ? re : (n < 8 ? -im : im);
		uint32_t hi, lo;
		tf32_split(v, hi, lo);
		b[umma_b_off(n, k)] = __uint_as_float(hi);
		b[umma_b_off(n + 16, k)] = __uint_as_float(lo);
	}
}

template <int SW>
__global__ void __launch_bounds__(256, 2)
	k_sweep_tm(const float2 *__restrict__ in, float2 *out, const unsigned char *__restrict__ prog,
		   double *partials, int pre)
{
	typedef float2 C2;
	constexpr int M = 12;
	extern __shared__ __align__(16) unsigned char sm[];
	const dk_sweep_hdr *h = reinterpret_cast<const dk_sweep_hdr *>(prog);
	const int m = h->m; /* == 12 (checked by the launcher) */
	const int lanes = m - PB;
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	const uint32_t wg = warp >> 2; /* warpgroup: row blocks 2 wg, 2 wg + 1 */
	const int npass = h->npass, ngate = h->ngate;
	const uint32_t tn_amp = 1u << M;
	const int ncond = (int)h->ncond;
	const size_t gate_bytes = (size_t)ngate * sizeof(dk_gate_desc);
	const size_t cond_bytes = (size_t)ncond * sizeof(dk_gate_cond);
	const int nmat = (int)((h->bytes - h->mat_off) / 16); /* complex entries */
	/* dynamic shared memory: two tile buffers (the next tile streams in
	 * while this one is processed), the gate list and conditions, the pass
	 * descriptors, and at a 1 KiB offset the matrices: every B' of the
	 * sweep (pre != 0) or the matrices in float2 for a per-entry B' */
	C2 *const bufs = reinterpret_cast<C2 *>(sm);
	uint4 *sg = reinterpret_cast<uint4 *>(sm + 2 * sizeof(C2) * tn_amp);
	dk_gate_cond *scond =
		reinterpret_cast<dk_gate_cond *>(reinterpret_cast<unsigned char *>(sg) + gate_bytes);
	dk_pass_desc *passes = reinterpret_cast<dk_pass_desc *>(
		reinterpret_cast<unsigned char *>(scond) + cond_bytes);
	const size_t mats_at =
		(2 * sizeof(C2) * tn_amp + gate_bytes + cond_bytes +
		 (size_t)npass * sizeof(dk_pass_desc) + 1023) & ~(size_t)1023;
	float *const mats_b = reinterpret_cast<float *>(sm + mats_at);
	float2 *const mats = reinterpret_cast<float2 *>(sm + mats_at);
	__shared__ __align__(1024) float sB[kTmBFloats]; /* per-entry B' */
	__shared__ __align__(8) uint64_t mbar[2];
	__shared__ uint32_t tslot;
	__shared__ uint8_t sq[16];
	__shared__ uint64_t soff[NA];
	__shared__ uint32_t sro[NA];
	__shared__ uint64_t sdep[DK_DEP_NIBBLES][16];

	{
		const uint4 *src = reinterpret_cast<const uint4 *>(prog + h->gate_off);
		for (int i = tid; i < ngate; i += blockDim.x)
			sg[i] = __ldg(src + i);
		const uint4 *csrc = reinterpret_cast<const uint4 *>(prog + h->cond_off);
		uint4 *cdst = reinterpret_cast<uint4 *>(scond);
		for (int i = tid; i < ncond; i += blockDim.x)
			cdst[i] = __ldg(csrc + i);
		const uint4 *psrc = reinterpret_cast<const uint4 *>(prog + h->pass_off);
		uint4 *pdst = reinterpret_cast<uint4 *>(passes);
		const int pwords = npass * (int)(sizeof(dk_pass_desc) / 16);
		for (int i = tid; i < pwords; i += blockDim.x)
			pdst[i] = __ldg(psrc + i);
		const double2 *msrc = reinterpret_cast<const double2 *>(prog + h->mat_off);
		if (pre) {
			for (int mi = 0; 64 * mi < nmat; ++mi)
				tm_write_b(mats_b + (size_t)kTmBFloats * mi, msrc + 64 * mi, (int)tid,
					   (int)blockDim.x);
			/* read by the tensor cores (async proxy) */
			asm volatile("fence.proxy.async.shared::cta;" ::);
		} else {
			for (int i = tid; i < nmat; i += blockDim.x) {
				const double2 v = __ldg(msrc + i);
				mats[i] = make_float2((float)v.x, (float)v.y);
			}
		}
		for (int i = tid; i < 16; i += blockDim.x)
			sq[i] = h->qpos[i];
	}
	if (tid == 0) {
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
		asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
		asm volatile("fence.mbarrier_init.release.cluster;" ::);
	}
	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
				     smem_u32(&tslot)),
			     "r"(kTmCols));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::);
	__syncthreads();
	asm volatile("tcgen05.fence::after_thread_sync;" ::);
	const uint32_t tbase = tslot;
	for (int r = tid; r < NA; r += blockDim.x) {
		uint64_t o = 0;
		for (int j = 0; j < PB; ++j)
			if ((r >> j) & 1)
				o |= 1ull << sq[lanes + j];
		soff[r] = o;
		sro[r] = swz_map((uint32_t)r << lanes, h->bankv);
	}
	for (int e = tid; e < DK_DEP_NIBBLES * 16; e += blockDim.x) {
		uint64_t v = (uint64_t)(e & 15) << (4 * (e >> 4));
		for (int j = 0; j < m; ++j) {
			const int q = sq[j];
			v = ((v >> q) << (q + 1)) | (v & ((1ull << q) - 1ull));
		}
		sdep[e >> 4][e & 15] = v;
	}
	/* streaming: thread t owns tile columns t and t + 256 (as k_sweep_tc) */
	uint64_t off_t0 = 0;
	for (int j = 0; j < lanes; ++j)
		if ((tid >> j) & 1u)
			off_t0 |= 1ull << sq[j];
	const uint32_t stid0 = swz_map(tid, h->bankv);
	const uint32_t s256 = swz_map(256u, h->bankv);
	auto off_t = [&](int hh) -> uint64_t { return hh ? (off_t0 | (1ull << sq[8])) : off_t0; };
	auto stid = [&](int hh) -> uint32_t { return hh ? (stid0 ^ s256) : stid0; };
	/* passes: this thread's columns, one per row block it owns */
	const uint32_t rb0 = 2u * wg;
	uint32_t col[2];
	col[0] = 128u * rb0 + 32u * (warp & 3u) + lane;
	col[1] = col[0] + 128u;
	const uint32_t ta = tbase + ((32u * (warp & 3u)) << 16); /* this warp's lane quarter */
	const uint32_t mb = smem_u32(&mbar[wg]);
	const bool issuer = tid == 128u * wg;
	__syncthreads();
	const uint64_t ntiles = h->ntiles;
	const int ndep = (h->n - m + 3) >> 2;
	const bool skip_idle = (in == out) && !h->all_touched;

	auto tile_base = [&](uint64_t t) -> uint64_t {
		uint64_t base = 0;
#pragma unroll
		for (int k = 0; k < DK_DEP_NIBBLES; ++k)
			if (k < ndep)
				base |= sdep[k][(t >> (4 * k)) & 15u];
		return base;
	};
	auto next_tile = [&](uint64_t t) -> uint64_t {
		for (; t < ntiles; t += gridDim.x) {
			if (!skip_idle)
				return t;
			const uint64_t base = tile_base(t);
			for (int g = 0; g < ngate; ++g) {
				const uint32_t gi = sg[g].y & 0xffffu;
				if (gi == 0xffffu)
					return t;
				const dk_gate_cond c = scond[gi];
				if (((base & c.gc) == c.gc) && !(base & c.ga))
					return t;
			}
		}
		return ntiles;
	};
	[[maybe_unused]] const uint64_t nglob = 1ull << h->n;
	auto prefetch = [&](uint64_t base, C2 *tile) {
#pragma unroll
		for (int hh = 0; hh < 2; ++hh) {
			const uint64_t bo = base | off_t(hh);
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t so = stid(hh) ^ sro[r];
				const uint64_t gi = bo | soff[r];
				if (!DK_IN_BOUNDS(so, tn_amp, CHK_LOAD_SMEM) ||
				    !DK_IN_BOUNDS(gi, nglob, CHK_LOAD_GLOBAL))
					continue;
				cp_async8(tile + so, in + gi);
			}
		}
		cp_async_commit();
	};

	double insq = 0.0, outsq = 0.0;
	uint32_t phase = 0; /* of this warpgroup's mbarrier */
	bool fault = false;
	uint64_t t = next_tile(blockIdx.x);
	if (t < ntiles)
		prefetch(tile_base(t), bufs);
	int cur = 0;
	while (t < ntiles && !fault) {
		const uint64_t base = tile_base(t);
		C2 *const tile = bufs + (size_t)cur * tn_amp;
		cp_async_wait_all();
		__syncthreads();
		/* the next tile streams into the other buffer (read out, and the
		 * barrier above passed, one tile ago) while this one is processed */
		const uint64_t tn = next_tile(t + gridDim.x);
		if (tn < ntiles)
			prefetch(tile_base(tn), bufs + (size_t)(cur ^ 1) * tn_amp);
		if (skip_idle) {
#pragma unroll
			for (int hh = 0; hh < 2; ++hh)
#pragma unroll
				for (int r = 0; r < NA; ++r) {
					const uint32_t so = stid(hh) ^ sro[r];
					if (DK_IN_BOUNDS(so, tn_amp, CHK_READOUT))
						insq += sqabs(tile[so]);
				}
			__syncthreads();
		}
		for (int p = 0; p < npass && !fault; ++p) {
			const dk_pass_desc *pd = passes + p;
			const uint32_t s0 = pd->sp[0], s1 = pd->sp[1], s2 = pd->sp[2];
			uint32_t cs[2];
#pragma unroll
			for (int j = 0; j < 2; ++j)
				cs[j] = pd->slo[col[j] & 31u] ^ pd->shi[col[j] >> 5];
			const int g1 = pd->g1;
			for (int g = pd->g0; g < g1; ++g) {
				const uint4 d = sg[g];
				const uint32_t gi = d.y & 0xffffu;
				if (gi != 0xffffu) {
					const dk_gate_cond c = scond[gi];
					if (((base & c.gc) != c.gc) || (base & c.ga))
						continue; /* the same for every thread */
				}
				const uint32_t mi = tc_matrix(d, scond, base);
				uint32_t bsm;
				if (pre) {
					bsm = smem_u32(mats_b + (size_t)kTmBFloats * mi);
				} else {
					/* B' of this entry; the previous entry's MMAs were
					 * waited for before the barrier that ended it */
					tm_write_b(sB, mats + 64 * (size_t)mi, (int)tid, (int)blockDim.x);
					asm volatile("fence.proxy.async.shared::cta;" ::);
					bsm = smem_u32(sB);
				}
#pragma unroll
				for (int j = 0; j < 2; ++j) {
					uint32_t vh[16], vl[16];
#pragma unroll
					for (int r = 0; r < NA; ++r) {
						const uint32_t so = cs[j] ^ ((r & 1) ? s0 : 0u) ^
								    ((r & 2) ? s1 : 0u) ^ ((r & 4) ? s2 : 0u);
						const C2 x = DK_IN_BOUNDS(so, tn_amp, CHK_GATHER) ? tile[so] : C2{};
						tf32_split(x.x, vh[r], vl[r]);
						tf32_split(x.y, vh[8 + r], vl[8 + r]);
					}
					const uint32_t rb = rb0 + (uint32_t)j;
					tm_st16(ta + 16u * rb, vh);
					tm_st16(ta + 64u + 16u * rb, vl);
				}
				asm volatile("tcgen05.wait::st.sync.aligned;" ::);
				asm volatile("tcgen05.fence::before_thread_sync;" ::);
				/* this warpgroup's rows are in tensor memory (and, per
				 * entry, B' in shared memory: then the whole CTA) */
				if (!pre)
					__syncthreads();
				else if (wg == 0)
					asm volatile("bar.sync 1, 128;" ::: "memory");
				else
					asm volatile("bar.sync 2, 128;" ::: "memory");
				if (issuer && !DK_TM_STARVED()) {
					asm volatile("tcgen05.fence::after_thread_sync;" ::);
					const uint64_t b0 = umma_desc_k(bsm), b1 = umma_desc_k(bsm + 1024u);
#pragma unroll
					for (uint32_t rb = rb0; rb < rb0 + 2u; ++rb) {
						const uint32_t dcol = tbase + 128u + 32u * rb;
						const uint32_t ah = tbase + 16u * rb, al = tbase + 64u + 16u * rb;
						/* hi*hi -> D[0, 16), hi*lo -> D[16, 32) */
						umma_tf32_ts(dcol, ah, b0, kTmIdesc32, 0u);
						umma_tf32_ts(dcol, ah + 8u, b1, kTmIdesc32, 1u);
						/* lo*hi -> D[16, 32) (B' rows 0..15 = R_hi) */
						umma_tf32_ts(dcol + 16u, al, b0, kTmIdesc16, 1u);
						umma_tf32_ts(dcol + 16u, al + 8u, b1, kTmIdesc16, 1u);
					}
					asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
						     ::"r"(mb));
				}
				const bool ok = tm_wait(mb, phase);
				phase ^= 1u;
				asm volatile("tcgen05.fence::after_thread_sync;" ::);
				const bool ctl = (d.x & 0xffffu) == DK_GC_DENSE3 + 1;
#pragma unroll
				for (int j = 0; j < 2; ++j) {
					/* both loads while the warp is converged
					 * (.sync.aligned), before any per-column branch */
					uint32_t yh[16], yc[16];
					const uint32_t dcol = ta + 128u + 32u * (rb0 + (uint32_t)j);
					tm_ld16(dcol, yh);
					tm_ld16(dcol + 16u, yc);
					asm volatile("tcgen05.wait::ld.sync.aligned;" ::);
					if (!ok)
						continue;
					if (ctl) { /* rare: controls off the pass bits */
						const uint32_t raw = pd->rlo[col[j] & 31u] | pd->rhi[col[j] >> 5];
						if (!ctl_ok(raw, d.z, d.w))
							continue;
					}
#pragma unroll
					for (int r = 0; r < NA; ++r) {
						const uint32_t so = cs[j] ^ ((r & 1) ? s0 : 0u) ^
								    ((r & 2) ? s1 : 0u) ^ ((r & 4) ? s2 : 0u);
						if (DK_IN_BOUNDS(so, tn_amp, CHK_SCATTER))
							tile[so] = make_float2(
								__uint_as_float(yh[r]) + __uint_as_float(yc[r]),
								__uint_as_float(yh[8 + r]) +
									__uint_as_float(yc[8 + r]));
					}
				}
				/* the scatters precede the next gather and B' rewrite;
				 * a timeout anywhere stops every thread */
				asm volatile("tcgen05.fence::before_thread_sync;" ::);
				if (__syncthreads_or(!ok)) {
					fault = true;
					break;
				}
			}
		}
		if (fault)
			break;
#pragma unroll
		for (int hh = 0; hh < 2; ++hh) {
			const uint64_t bo = base | off_t(hh);
#pragma unroll
			for (int r = 0; r < NA; ++r) {
				const uint32_t so = stid(hh) ^ sro[r];
				const C2 v = DK_IN_BOUNDS(so, tn_amp, CHK_READOUT) ? tile[so] : C2{};
				outsq += sqabs(v);
				if (DK_IN_BOUNDS(bo | soff[r], nglob, CHK_STORE))
					__stcs(out + (bo | soff[r]), v);
			}
		}
		t = tn;
		cur ^= 1;
	}
	cp_async_wait_all();
	if (fault) {
		/* the MMAs of an expired wait may still run: give each
		 * warpgroup's another bounded wait before the tensor memory is
		 * released */
		if (issuer) {
			if (tid == 0)
				atomicAdd(&g_dk_tm_fault, 1u);
			(void)tm_wait(mb, phase ^ 1u);
		}
		insq = outsq = __longlong_as_double(0x7ff8000000000000ll);
	}
	asm volatile("tcgen05.fence::before_thread_sync;" ::);
	__syncthreads();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase),
			     "r"(kTmCols));
	block_sum2(insq, outsq);
	if (tid == 0) {
		partials[2 * blockIdx.x] = insq;
		partials[2 * blockIdx.x + 1] = outsq;
	}
}

enum { FIN_GATE = 0, FIN_COLLAPSE = 1, FIN_RESET = 2 };

/* Sum the (in, out) partials of `nb` blocks in a fixed order and update the
 * output scalars.  FIN_GATE: csq = all ? out : csq_in - in + out, norm =
 * sqrt(csq).  FIN_COLLAPSE: csq = out, norm = norm_in * sqrt(p_sel).
 * FIN_RESET: csq = out, norm = 1. */
__global__ void k_finalize(const double *partials, int nb, const dk_scal *sc_in,
			   dk_scal *sc_out, int mode, int all)
{
	__shared__ double sx[256], sy[256];
	double x = 0.0, y = 0.0;
	for (int i = threadIdx.x; i < nb; i += blockDim.x) {
		x += partials[2 * i];
		y += partials[2 * i + 1];
	}
	sx[threadIdx.x] = x;
	sy[threadIdx.x] = y;
	__syncthreads();
	for (int s = blockDim.x >> 1; s > 0; s >>= 1) {
		if ((int)threadIdx.x < s) {
			sx[threadIdx.x] += sx[threadIdx.x + s];
			sy[threadIdx.x] += sy[threadIdx.x + s];
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		const double sin_ = sx[0], sout = sy[0];
		if (mode == FIN_GATE) {
			const double c = all ? sout : (sc_in->csq - sin_ + sout);
			sc_out->csq = c;
			sc_out->norm = sqrt(c);
		} else if (mode == FIN_COLLAPSE) {
			const double nrm = sc_in->norm * sqrt(sc_out->p_sel);
			sc_out->csq = sout;
			sc_out->norm = nrm;
			if (nrm == 0.0)
				sc_out->zero_norm = 1;
		} else {
			sc_out->csq = sout;
			sc_out->norm = 1.0;
		}
	}
}

/* ---- generic single gate (any k), out of place ----------------------- */

struct GenTargets {
	uint8_t t[DK_MAX_GATE_QUBITS];
};

template <typename R>
__global__ void __launch_bounds__(256)
	k_generic(const typename CT<R>::T *__restrict__ in, typename CT<R>::T *out,
		  uint64_t size, int k, GenTargets tg, uint64_t cm, uint64_t am,
		  const double2 *__restrict__ mat, double *partials)
{
	typedef typename CT<R>::T C2;
	uint64_t tmask = 0;
	for (int j = 0; j < k; ++j)
		tmask |= 1ull << tg.t[j];
	const uint32_t dim = 1u << k;
	double outsq = 0.0, dummy = 0.0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
	     i += (uint64_t)gridDim.x * blockDim.x) {
		C2 v;
		if ((i & cm) == cm && !(i & am)) {
			uint32_t row = 0;
			for (int j = 0; j < k; ++j)
				row |= (uint32_t)((i >> tg.t[j]) & 1u) << j;
			const uint64_t clr = i & ~tmask;
			double2 acc = make_double2(0.0, 0.0);
			for (uint32_t col = 0; col < dim; ++col) {
				uint64_t src = clr;
				for (int j = 0; j < k; ++j)
					src |= (uint64_t)((col >> j) & 1u) << tg.t[j];
				acc = cmad(__ldg(mat + (uint64_t)row * dim + col),
					   to_c128(in[src]), acc);
			}
			v = from_c128<C2>(acc);
		} else {
			v = in[i];
		}
		out[i] = v;
		outsq += sqabs(v);
	}
	block_sum2(dummy, outsq);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = outsq;
	}
}

/* ---- initialisation / import ------------------------------------------ */

template <typename R>
__global__ void k_set_one(typename CT<R>::T *d, dk_scal *sc)
{
	d[0] = mk((R)1, (R)0);
	sc->norm = 1.0;
	sc->csq = 1.0;
	sc->p_sel = 0.0;
	sc->flag = 0;
	sc->zero_norm = 0;
}

template <typename R>
__global__ void __launch_bounds__(256)
	k_import(const double2 *__restrict__ src, typename CT<R>::T *dst,
		 uint64_t size, double *partials)
{
	typedef typename CT<R>::T C2;
	double s = 0.0, dummy = 0.0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
	     i += (uint64_t)gridDim.x * blockDim.x) {
		const C2 v = from_c128<C2>(src[i]);
		dst[i] = v;
		s += sqabs(v);
	}
	block_sum2(dummy, s);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = s;
	}
}

/* Half of a register for an exchange between ranks (distributed registers):
 * dst[j] = scale * in[i(j)], i(j) = j with `value` inserted at bit `bit`,
 * for the 2^(n-1) indices j in order. */
template <typename R>
__global__ void __launch_bounds__(256)
	k_read_half(const typename CT<R>::T *__restrict__ in, uint64_t half, unsigned bit,
		    int value, double scale, typename CT<R>::T *dst)
{
	typedef typename CT<R>::T C2;
	const uint64_t low = (1ull << bit) - 1ull;
	for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < half;
	     j += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t i = ((j & ~low) << 1) | ((uint64_t)value << bit) | (j & low);
		const double2 v = to_c128(in[i]);
		dst[j] = from_c128<C2>(make_double2(v.x * scale, v.y * scale));
	}
}

/* The register with its half at bit `bit` = `value` replaced:
 * out[i] = src[j(i)] there (j(i) = i with bit `bit` removed), scale * in[i]
 * elsewhere; per-block sums of |out|^2 for the new register's scalars. */
template <typename R>
__global__ void __launch_bounds__(256)
	k_replace_half(const typename CT<R>::T *__restrict__ in,
		       const typename CT<R>::T *__restrict__ src, uint64_t size, unsigned bit,
		       int value, double scale, typename CT<R>::T *out, double *partials)
{
	typedef typename CT<R>::T C2;
	const uint64_t low = (1ull << bit) - 1ull;
	double sq = 0.0, dummy = 0.0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
	     i += (uint64_t)gridDim.x * blockDim.x) {
		C2 v;
		if ((int)((i >> bit) & 1ull) == value) {
			v = src[((i >> 1) & ~low) | (i & low)];
		} else {
			const double2 x = to_c128(in[i]);
			v = from_c128<C2>(make_double2(x.x * scale, x.y * scale));
		}
		out[i] = v;
		sq += sqabs(v);
	}
	block_sum2(dummy, sq);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = sq;
	}
}

__global__ void k_clear_flags(dk_scal *sc)
{
	sc->zero_norm = 0;
	sc->flag = 0;
	sc->p_sel = 0.0;
}

/* ---- marginals: S_q = sum_{bit q of i set} |amp_i|^2 for all q --------
 * Thread g visits i = (k << s) | g, s = log2(total threads): bits below s are
 * fixed per thread, bits above vary with k and are accumulated per bit in
 * acc[NB] (NB >= n - s, indexed only by unrolled constants so that it stays
 * in registers).  Two 256-thread blocks fit per SM. */
constexpr int kMargHi = 24;

/* Block sum of v into partials[slot] (thread 0), uniform call sites only. */
__device__ __forceinline__ void marg_store(double v, double *red, double *dst)
{
	const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	if (l == 0)
		red[w] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
			t += red[i];
		*dst = t;
	}
	__syncthreads();
}

template <typename R, int NB>
__global__ void __launch_bounds__(256, 2)
	k_marginals(const typename CT<R>::T *__restrict__ d, int n, int s,
		    double *partials)
{
	const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const int nb = n - s;
	/* registers smaller than one warp: lanes past the register stay idle */
	const uint64_t cnt = (g >> s) ? 0ull : (1ull << nb);
	double tot = 0.0;
	double acc[NB];
#pragma unroll
	for (int j = 0; j < NB; ++j)
		acc[j] = 0.0;
	if (cnt >= 16) {
		/* 16 consecutive k at a time: the 4 low bits of k take fixed
		 * patterns, every higher bit is constant over the group */
		for (uint64_t k0 = 0; k0 < cnt; k0 += 16) {
			double p[16];
#pragma unroll
			for (int e = 0; e < 16; ++e)
				p[e] = sqabs(__ldcs(d + (((k0 + e) << s) | g)));
			double t = 0.0;
#pragma unroll
			for (int e = 0; e < 16; ++e)
				t += p[e];
#pragma unroll
			for (int j = 0; j < 4; ++j) {
				double h = 0.0;
#pragma unroll
				for (int e = 0; e < 16; ++e)
					if ((e >> j) & 1)
						h += p[e];
				acc[j] += h;
			}
#pragma unroll
			for (int j = 4; j < NB; ++j)
				if (j < nb && ((k0 >> j) & 1u))
					acc[j] += t;
			tot += t;
		}
	} else {
		for (uint64_t k = 0; k < cnt; ++k) {
			const double p = sqabs(__ldcs(d + ((k << s) | g)));
			tot += p;
#pragma unroll
			for (int j = 0; j < NB; ++j)
				if (j < nb && ((k >> j) & 1u))
					acc[j] += p;
		}
	}
	__shared__ double red[32];
	double *const out = partials + (size_t)blockIdx.x * kPartialStride;
	/* q < s: tot * bit_q(g); q = s + j: acc[j]; q = n: tot */
	for (int q = 0; q < s && q < n; ++q)
		marg_store(((g >> q) & 1u) ? tot : 0.0, red, out + q);
#pragma unroll
	for (int j = 0; j < NB; ++j)
		if (j < nb)
			marg_store(acc[j], red, out + s + j);
	marg_store(tot, red, out + n);
}

__global__ void k_marg_finalize(const double *partials, int nb, int n, double *marg)
{
	const int q = threadIdx.x;
	if (q > n)
		return;
	double t = 0.0;
	for (int b = 0; b < nb; ++b)
		t += partials[(size_t)b * kPartialStride + q];
	marg[q] = t;
}

/* ---- measurement -------------------------------------------------------- */

/* qops.c:124-136: P(1) = S_q / norm^2 (the reference sums |amp/norm|^2);
 * result = P(1) > roll (or the forced value); keep the selected probability. */
__global__ void k_decide(const double *marg, int q, double roll, int forced,
			 const dk_scal *sc_in, dk_scal *sc_out)
{
	const double nrm = sc_in->norm;
	const double p1 = marg[q] / (nrm * nrm);
	const int res = forced >= 0 ? forced : (p1 > roll ? 1 : 0);
	sc_out->flag = res;
	sc_out->p_sel = res ? p1 : 1.0 - p1;
	sc_out->zero_norm = 0;
}

/* qops.c:138-174: out[j] = in[insert bit q = outcome into j] */
template <typename R>
__global__ void __launch_bounds__(256)
	k_collapse(const typename CT<R>::T *__restrict__ in, typename CT<R>::T *out,
		   uint64_t half, int q, const dk_scal *sc_sel, double *partials)
{
	typedef typename CT<R>::T C2;
	const uint64_t v = (uint64_t)sc_sel->flag << q;
	const uint64_t low = (1ull << q) - 1ull;
	double s = 0.0, dummy = 0.0;
	for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < half;
	     j += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t i = ((j & ~low) << 1) | v | (j & low);
		const C2 x = DK_IN_BOUNDS(i, 2 * half, CHK_COLLAPSE) ? __ldcs(in + i) : C2{};
		__stcs(out + j, x);
		s += sqabs(x);
	}
	block_sum2(dummy, s);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = s;
	}
}

/* ---- joint measurement of several qubits -------------------------------
 * The reference measures the masked qubits one after the other, highest
 * first (doki.c:1097-1157): p = P(q = 1) of the register collapsed so far,
 * outcome = p > roll, collapse and renormalise.  Equivalently, with the
 * joint distribution J over the k measured qubits (one pass over the
 * state), each p is the conditional S1 / S_prev of the outcomes decided so
 * far, and one gather applies all k collapses. */

/* index of the j-th amplitude whose measured bits are zero: j's bits
 * deposited into the unmeasured positions, one run of positions at a time */
struct DepRuns {
	uint8_t src[DK_MAX_QUBITS + 1], dst[DK_MAX_QUBITS + 1], len[DK_MAX_QUBITS + 1];
	int nruns;
};

__device__ __forceinline__ uint64_t dep_runs(const DepRuns &r, uint64_t j)
{
	uint64_t i = 0;
	for (int k = 0; k < r.nruns; ++k)
		i |= ((j >> r.src[k]) & ((1ull << r.len[k]) - 1ull)) << r.dst[k];
	return i;
}

__device__ __forceinline__ uint64_t deposit_mask(uint64_t v, uint64_t mask)
{
	uint64_t out = 0;
	for (int b = 0; mask; ++b) {
		const uint64_t low = mask & (~mask + 1ull);
		if ((v >> b) & 1ull)
			out |= low;
		mask &= mask - 1ull;
	}
	return out;
}

/* partials[bin * nchunk + c] = sum of |amp|^2 over chunk c of the bin */
template <typename R>
__global__ void __launch_bounds__(256)
	k_joint(const typename CT<R>::T *__restrict__ in, DepRuns runs, uint64_t mask,
		uint64_t per_bin, uint64_t chunk, uint64_t nchunk, double *partials)
{
	__shared__ DepRuns sr;
	if (threadIdx.x == 0)
		sr = runs;
	__syncthreads();
	const uint64_t bin = blockIdx.y;
	const uint64_t vb = deposit_mask(bin, mask);
	[[maybe_unused]] const uint64_t nin = per_bin << __popcll(mask);
	for (uint64_t c = blockIdx.x; c < nchunk; c += gridDim.x) {
		double sum = 0.0, dummy = 0.0;
		const uint64_t j0 = c * chunk;
		uint64_t j1 = j0 + chunk;
		if (j1 > per_bin)
			j1 = per_bin;
		for (uint64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
			const uint64_t i = dep_runs(sr, j) | vb;
			if (DK_IN_BOUNDS(i, nin, CHK_JOINT))
				sum += sqabs(__ldcs(in + i));
		}
		block_sum2(dummy, sum);
		if (threadIdx.x == 0)
			partials[bin * nchunk + c] = sum;
		__syncthreads();
	}
}

/* Joint distribution of k <= 4 measured qubits in one contiguous pass over
 * the register (coalesced like k_marginals): thread t adds |amp_i|^2 to its
 * own shared-memory column hist[bin(i)][t], no atomics, and the columns of
 * each bin are added in a fixed order.  Writes partials[bin * gridDim.x +
 * block] as k_joint does, for k_joint_finalize.  k_joint instead gives each
 * bin its own blocks, which gather the bin's amplitudes; with a low measured
 * qubit those gathers use part of every 32-byte sector and every bin re-reads
 * the same sectors. */
constexpr int kJointSmallBins = 16;
constexpr uint64_t kJointSeg = 4096; /* amplitudes per block step, 16 per thread */

template <typename R>
__global__ void __launch_bounds__(256)
	k_joint_small(const typename CT<R>::T *__restrict__ in, uint64_t size, uint32_t qpack,
		      int k, double *partials)
{
	__shared__ double hist[kJointSmallBins][256];
	const uint32_t t = threadIdx.x;
	const int nb = 1 << k;
	for (int b = 0; b < nb; ++b)
		hist[b][t] = 0.0; /* each thread only ever touches its own column */
	int qs[4];
#pragma unroll
	for (int j = 0; j < 4; ++j)
		qs[j] = (int)((qpack >> (8 * j)) & 0xffu);
	for (uint64_t base = (uint64_t)blockIdx.x * kJointSeg; base < size;
	     base += (uint64_t)gridDim.x * kJointSeg) {
		double p[16];
#pragma unroll
		for (int u = 0; u < 16; ++u)
			p[u] = DK_IN_BOUNDS(base + t + 256u * u, size, CHK_JOINT)
				       ? sqabs(__ldcs(in + base + t + 256u * u))
				       : 0.0;
#pragma unroll
		for (int u = 0; u < 16; ++u) {
			const uint64_t i = base + t + 256u * u;
			uint32_t b = 0;
#pragma unroll
			for (int j = 0; j < 4; ++j)
				if (j < k)
					b |= (uint32_t)((i >> qs[j]) & 1u) << j;
			hist[b][t] += p[u];
		}
	}
	__syncthreads();
	const uint32_t w = t >> 5, l = t & 31u;
	for (int b = (int)w; b < nb; b += (int)(blockDim.x >> 5)) {
		double v = 0.0;
		for (uint32_t c = l; c < 256u; c += 32u)
			v += hist[b][c];
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			v += __shfl_xor_sync(0xffffffffu, v, o);
		if (l == 0)
			partials[(uint64_t)b * gridDim.x + blockIdx.x] = v;
	}
}

/* joint[bin] = sum of its chunks, in order */
__global__ void __launch_bounds__(256)
	k_joint_finalize(const double *partials, uint64_t nchunk, double *joint)
{
	double sum = 0.0, dummy = 0.0;
	for (uint64_t c = threadIdx.x; c < nchunk; c += blockDim.x)
		sum += partials[blockIdx.x * nchunk + c];
	block_sum2(dummy, sum);
	if (threadIdx.x == 0)
		joint[blockIdx.x] = sum;
}

/* One warp: outcomes of the k measured qubits, highest first, from the
 * joint distribution; flags[s] = outcome of step s; *vbits = the outcomes
 * deposited into the measured positions; sc_out->p_sel = probability of the
 * whole outcome relative to the stored norm. */
__global__ void k_decide_joint(const double *joint, int k, const double *rolls, int32_t *flags,
			       uint64_t *vbits, uint64_t mask, const dk_scal *sc_in,
			       dk_scal *sc_out)
{
	const uint32_t lane = threadIdx.x;
	const uint32_t nb = 1u << k;
	/* the first probability is relative to the stored norm, as the
	 * reference's (data registers need not be normalised); the later ones
	 * are conditional on the outcomes so far */
	const double n2 = sc_in->norm * sc_in->norm;
	uint32_t pm = 0, pv = 0;
	double prev = n2;
	for (int st = 0; st < k; ++st) {
		const int bb = k - 1 - st; /* bin bit of the qubit measured now */
		double s1 = 0.0, s0 = 0.0;
		for (uint32_t b = lane; b < nb; b += 32)
			if ((b & pm) == pv) {
				if ((b >> bb) & 1u)
					s1 += joint[b];
				else
					s0 += joint[b];
			}
		for (int o = 16; o > 0; o >>= 1) {
			s1 += __shfl_xor_sync(0xffffffffu, s1, o);
			s0 += __shfl_xor_sync(0xffffffffu, s0, o);
		}
		const double p = prev > 0.0 ? s1 / prev : 0.0;
		const int res = p > rolls[st] ? 1 : 0;
		pm |= 1u << bb;
		pv |= (uint32_t)res << bb;
		prev = res ? s1 : s0;
		if (lane == 0)
			flags[st] = res;
	}
	if (lane == 0) {
		*vbits = deposit_mask(pv, mask);
		sc_out->flag = 0;
		sc_out->p_sel = n2 > 0.0 ? prev / n2 : 0.0;
		sc_out->zero_norm = 0;
	}
}

/* out[j] = in[j deposited into the unmeasured positions | measured bits] */
template <typename R>
__global__ void __launch_bounds__(256)
	k_collapse_joint(const typename CT<R>::T *__restrict__ in, typename CT<R>::T *out,
			 DepRuns runs, uint64_t size, const uint64_t *vbits, double *partials,
			 [[maybe_unused]] uint64_t in_size)
{
	typedef typename CT<R>::T C2;
	__shared__ DepRuns sr;
	if (threadIdx.x == 0)
		sr = runs;
	__syncthreads();
	const uint64_t v = *vbits;
	double s = 0.0, dummy = 0.0;
	for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < size;
	     j += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t i = dep_runs(sr, j) | v;
		const C2 x = DK_IN_BOUNDS(i, in_size, CHK_COLLAPSE) ? __ldcs(in + i) : C2{};
		__stcs(out + j, x);
		s += sqabs(x);
	}
	block_sum2(dummy, s);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = s;
	}
}

/* ---- join (qops.c:97-122) ---------------------------------------------- */
template <typename R>
__global__ void __launch_bounds__(256)
	k_join(const typename CT<R>::T *__restrict__ most, const dk_scal *sc1,
	       const typename CT<R>::T *__restrict__ least, const dk_scal *sc2,
	       int n2, typename CT<R>::T *out, uint64_t size, double *partials)
{
	typedef typename CT<R>::T C2;
	const double i1 = 1.0 / sc1->norm, i2 = 1.0 / sc2->norm;
	const uint64_t lm = (1ull << n2) - 1ull;
	double s = 0.0, dummy = 0.0;
	for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < size;
	     o += (uint64_t)gridDim.x * blockDim.x) {
		const double2 a = to_c128(most[o >> n2]);
		const double2 b = to_c128(__ldg(least + (o & lm)));
		const double2 an = make_double2(a.x * i1, a.y * i1);
		const double2 bn = make_double2(b.x * i2, b.y * i2);
		const C2 v = from_c128<C2>(cmul(an, bn));
		__stcs(out + o, v);
		s += sqabs(v);
	}
	block_sum2(dummy, s);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = s;
	}
}

/* Join with a least register larger than the L2 and a small most register:
 * one thread per least amplitude, read once, times every most amplitude
 * (k_join above re-reads the whole least register once per most amplitude).
 * Same products as k_join; writes are coalesced over consecutive l. */
template <typename R>
__global__ void __launch_bounds__(256)
	k_join_wide(const typename CT<R>::T *__restrict__ most, const dk_scal *sc1,
		    const typename CT<R>::T *__restrict__ least, const dk_scal *sc2, int n1,
		    int n2, typename CT<R>::T *out, double *partials)
{
	typedef typename CT<R>::T C2;
	const double i1 = 1.0 / sc1->norm, i2 = 1.0 / sc2->norm;
	const uint64_t nl = 1ull << n2, nm = 1ull << n1;
	double s = 0.0, dummy = 0.0;
	for (uint64_t l = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nl;
	     l += (uint64_t)gridDim.x * blockDim.x) {
		const double2 b = to_c128(__ldcs(least + l));
		const double2 bn = make_double2(b.x * i2, b.y * i2);
		for (uint64_t m = 0; m < nm; ++m) {
			const double2 a = to_c128(__ldg(most + m));
			const double2 an = make_double2(a.x * i1, a.y * i1);
			const C2 v = from_c128<C2>(cmul(an, bn));
			__stcs(out + ((m << n2) | l), v);
			s += sqabs(v);
		}
	}
	block_sum2(dummy, s);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = 0.0;
		partials[2 * blockIdx.x + 1] = s;
	}
}

/* ---- first non-zero amplitude (qops.c:57-65) ---------------------------- */
template <typename R>
__global__ void __launch_bounds__(256)
	k_first_nz(const typename CT<R>::T *__restrict__ d, uint64_t first,
		   uint64_t count, unsigned long long *res)
{
	unsigned long long best = ~0ull;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
	     i += (uint64_t)gridDim.x * blockDim.x) {
		const typename CT<R>::T v = d[first + i];
		if (v.x != 0 || v.y != 0) {
			best = first + i;
			break; /* later i of this thread are larger */
		}
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) {
		const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
		best = x < best ? x : best;
	}
	if ((threadIdx.x & 31) == 0 && best != ~0ull)
		atomicMin(res, best);
}

/* ---- reduced density matrix helpers ------------------------------------ */
__device__ __forceinline__ uint64_t deposit(uint64_t v, uint64_t mask)
{
	uint64_t r = 0;
	for (uint64_t b = 1; mask; b <<= 1) {
		const uint64_t low = mask & (~mask + 1ull);
		if (v & b)
			r |= low;
		mask &= mask - 1ull;
	}
	return r;
}

template <typename R>
__global__ void __launch_bounds__(256)
	k_gather_kept(const typename CT<R>::T *__restrict__ d, uint64_t keep,
		      uint64_t trace, int k, uint64_t total, double2 *M)
{
	for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
	     e += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t a = e & ((1ull << k) - 1ull), b = e >> k;
		M[e] = to_c128(d[deposit(a, keep) | deposit(b, trace)]);
	}
}

/* The gather above when the kept qubits are the low k ones: X is the
 * register itself, widened to FP64 -- two amplitudes per 16-byte load. */
__global__ void __launch_bounds__(256)
	k_widen_c64(const float4 *__restrict__ d, double4 *M, uint64_t pairs)
{
	for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < pairs;
	     e += (uint64_t)gridDim.x * blockDim.x) {
		const float4 v = __ldcs(d + e);
		M[e] = make_double4((double)v.x, (double)v.y, (double)v.z, (double)v.w);
	}
}

__global__ void __launch_bounds__(256)
	k_herm_fill(const double2 *__restrict__ C, double2 *rho, uint64_t dim)
{
	const uint64_t total = dim * dim;
	for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
	     e += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t a = e / dim, a2 = e % dim;
		double2 v;
		if (a >= a2)
			v = C[a + a2 * dim];
		else {
			v = C[a2 + a * dim];
			v.y = -v.y;
		}
		rho[e] = v;
	}
}

/* ---- reduced density matrix -------------------------------------------
 * rho = alpha X X^H, X[a][b] = A[b * dim + a] (a: kept index, b: traced
 * index), into the lower triangle of the column-major C (C[a + a' dim],
 * a >= a').  The traced index is split into nsplit chunks whose partial
 * products go to part[s] and are added in a fixed order by k_rho_reduce. */

constexpr int kRhoTile = 64; /* output tile (rows and columns) */
constexpr int kRhoSlab = 32; /* traced values per shared-memory slab */

__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, bool valid)
{
	const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem),
		     "r"(valid ? 16 : 0));
}

/* One lower 64x64 tile (ti >= tj) per CTA and one traced chunk per grid row.
 * 8 warps as 2 x 4: a warp owns rows 32 wr .. +32 (4 MMA row blocks) and
 * columns 16 wc .. +16 (2 column blocks).  Per 4 traced values (one k-step)
 * each 8x8 block takes 3 FP64 MMAs (Gauss): P1 += Xr Xr'^T, P2 += Xi Xi'^T,
 * P3 += (Xr + Xi)(Xr' - Xi')^T; re = P1 + P2, im = P3 - P1 + P2.  The 48
 * accumulators of a lane need one CTA per SM; slabs of 32 traced values
 * (128 KiB double-buffered) keep block barriers to one per 8 k-steps.
 * Slabs are stored [b][a ^ 2 (b & 3)] so a quarter-warp's fragment reads
 * (4 traced rows x 2 columns) hit 8 distinct 16-byte bank groups. */
__global__ void __launch_bounds__(256, 1)
	k_rho_tc(const double2 *__restrict__ A, uint64_t dim, uint64_t K, uint64_t bchunk,
		 double2 *part, double alpha)
{
	extern __shared__ __align__(16) unsigned char rsm[];
	/* [buffer][row tile, column tile][traced][kept] */
	double2 (*sab)[2][kRhoSlab][kRhoTile] =
		reinterpret_cast<double2 (*)[2][kRhoSlab][kRhoTile]>(rsm);
	const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
	const uint32_t g = lane >> 2, t = lane & 3u, wr = warp & 1u, wc = warp >> 1;
	/* lower-triangle tile index -> (ti, tj) */
	const uint64_t x = blockIdx.x;
	uint64_t ti = (uint64_t)((sqrt(8.0 * (double)x + 1.0) - 1.0) * 0.5);
	while ((ti + 1) * (ti + 2) / 2 <= x)
		++ti;
	while (ti * (ti + 1) / 2 > x)
		--ti;
	const uint64_t tj = x - ti * (ti + 1) / 2;
	const uint64_t a0 = ti * kRhoTile, c0 = tj * kRhoTile;
	const bool diag = ti == tj;
	const uint64_t b_begin = (uint64_t)blockIdx.y * bchunk;
	uint64_t b_end = b_begin + bchunk;
	if (b_end > K)
		b_end = K;

	auto load = [&](int buf, uint64_t b0) {
#pragma unroll
		for (int r = 0; r < (kRhoSlab * kRhoTile) / 256; ++r) {
			const uint32_t e = tid + 256u * r;
			const uint32_t bl = e / kRhoTile, al = e % kRhoTile;
			const uint64_t b = b0 + bl;
			const bool ok = b < b_end;
			const uint32_t pa = al ^ ((bl & 3u) << 1);
			cp_async16_zfill(&sab[buf][0][bl][pa], A + (ok ? b * dim + a0 + al : 0), ok);
			if (!diag)
				cp_async16_zfill(&sab[buf][1][bl][pa], A + (ok ? b * dim + c0 + al : 0),
						 ok);
		}
		cp_async_commit();
	};

	double acc[4][2][6]; /* Gauss: Xr Xr', Xi Xi', (Xr + Xi)(Xr' - Xi') */
#pragma unroll
	for (int i = 0; i < 4; ++i)
#pragma unroll
		for (int j = 0; j < 2; ++j)
#pragma unroll
			for (int v = 0; v < 6; ++v)
				acc[i][j][v] = 0.0;

	const int bsel = diag ? 0 : 1;
	int cur = 0;
	if (b_begin < b_end)
		load(0, b_begin);
	for (uint64_t b0 = b_begin; b0 < b_end; b0 += kRhoSlab) {
		if (b0 + kRhoSlab < b_end) {
			load(cur ^ 1, b0 + kRhoSlab);
			asm volatile("cp.async.wait_group 1;\n" ::);
		} else {
			cp_async_wait_all();
		}
		__syncthreads();
#pragma unroll
		for (int ks = 0; ks < kRhoSlab / 4; ++ks) {
			const uint32_t bl = 4u * ks + t;
			const uint32_t sw = (bl & 3u) << 1;
			double2 xa[4], xb[2];
#pragma unroll
			for (int i = 0; i < 4; ++i)
				xa[i] = sab[cur][0][bl][(32u * wr + 8u * i + g) ^ sw];
#pragma unroll
			for (int j = 0; j < 2; ++j)
				xb[j] = sab[cur][bsel][bl][(16u * wc + 8u * j + g) ^ sw];
#pragma unroll
			for (int i = 0; i < 4; ++i)
#pragma unroll
				for (int j = 0; j < 2; ++j) {
					dmma(acc[i][j][0], acc[i][j][1], xa[i].x, xb[j].x);
					dmma(acc[i][j][2], acc[i][j][3], xa[i].y, xb[j].y);
					dmma(acc[i][j][4], acc[i][j][5], xa[i].x + xa[i].y, xb[j].x - xb[j].y);
				}
		}
		__syncthreads(); /* this buffer is refilled two slabs later */
		cur ^= 1;
	}
	double2 *P = part + (uint64_t)blockIdx.y * dim * dim;
	const double f = gridDim.y == 1 ? alpha : 1.0;
#pragma unroll
	for (int i = 0; i < 4; ++i)
#pragma unroll
		for (int j = 0; j < 2; ++j)
#pragma unroll
			for (int e = 0; e < 2; ++e) {
				const uint64_t a = a0 + 32u * wr + 8u * i + g;
				const uint64_t c = c0 + 16u * wc + 8u * j + 2u * t + e;
				const double p1 = acc[i][j][e], p2 = acc[i][j][2 + e], p3 = acc[i][j][4 + e];
				P[a + c * dim] = make_double2(f * (p1 + p2), f * (p3 - p1 + p2));
			}
}

/* Kept sets below 64 amplitudes: one CTA per traced chunk stages the chunk
 * and every thread accumulates up to 4 of the dim^2 products. */
__global__ void __launch_bounds__(256)
	k_rho_small(const double2 *__restrict__ A, uint32_t dim, uint64_t K, uint64_t bchunk,
		    double2 *part)
{
	__shared__ double2 sx[2048];
	const uint32_t per = 2048u / dim; /* traced values per staging round */
	const uint64_t b_begin = (uint64_t)blockIdx.x * bchunk;
	uint64_t b_end = b_begin + bchunk;
	if (b_end > K)
		b_end = K;
	double re[4] = { 0.0, 0.0, 0.0, 0.0 }, im[4] = { 0.0, 0.0, 0.0, 0.0 };
	const uint32_t nout = dim * dim;
	for (uint64_t b0 = b_begin; b0 < b_end; b0 += per) {
		const uint64_t nb = (b_end - b0) < per ? (b_end - b0) : per;
		for (uint32_t e = threadIdx.x; e < nb * dim; e += blockDim.x)
			sx[e] = A[b0 * dim + e];
		__syncthreads();
#pragma unroll
		for (int r = 0; r < 4; ++r) {
			const uint32_t o = threadIdx.x + 256u * r;
			if (o >= nout)
				continue;
			const uint32_t a = o % dim, c = o / dim;
			for (uint32_t b = 0; b < nb; ++b) {
				const double2 u = sx[b * dim + a], v = sx[b * dim + c];
				re[r] = fma(u.x, v.x, fma(u.y, v.y, re[r]));
				im[r] = fma(u.y, v.x, fma(-u.x, v.y, im[r]));
			}
		}
		__syncthreads();
	}
	double2 *P = part + (uint64_t)blockIdx.x * nout;
#pragma unroll
	for (int r = 0; r < 4; ++r) {
		const uint32_t o = threadIdx.x + 256u * r;
		if (o < nout)
			P[o] = make_double2(re[r], im[r]);
	}
}

/* C = alpha * sum over s (in order) of part[s], on the lower tiles */
__global__ void __launch_bounds__(256)
	k_rho_reduce(const double2 *__restrict__ part, int nsplit, uint64_t dim, double alpha,
		     double2 *C)
{
	const uint64_t total = dim * dim;
	for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
	     e += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t a = e % dim, c = e / dim;
		if (a / kRhoTile < c / kRhoTile)
			continue;
		double x = 0.0, y = 0.0;
		for (int s2 = 0; s2 < nsplit; ++s2) {
			const double2 v = part[(uint64_t)s2 * total + e];
			x += v.x;
			y += v.y;
		}
		C[e] = make_double2(alpha * x, alpha * y);
	}
}

template <typename R>
__global__ void __launch_bounds__(256)
	k_rho_elem(const typename CT<R>::T *__restrict__ d, uint64_t ia, uint64_t ib,
		   uint64_t trace, uint64_t cnt, double *partials)
{
	double re = 0.0, im = 0.0;
	for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < cnt;
	     b += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t off = deposit(b, trace);
		const double2 x = to_c128(d[ia | off]), y = to_c128(d[ib | off]);
		/* x * conj(y) */
		re += x.x * y.x + x.y * y.y;
		im += x.y * y.x - x.x * y.y;
	}
	block_sum2(re, im);
	if (threadIdx.x == 0) {
		partials[2 * blockIdx.x] = re;
		partials[2 * blockIdx.x + 1] = im;
	}
}

__global__ void k_rho_elem_finalize(const double *partials, int nb,
				    const dk_scal *sc, double *outv)
{
	if (threadIdx.x != 0)
		return;
	double re = 0.0, im = 0.0;
	for (int b = 0; b < nb; ++b) {
		re += partials[2 * b];
		im += partials[2 * b + 1];
	}
	const double n2 = sc->norm * sc->norm;
	outv[0] = re / n2;
	outv[1] = im / n2;
}

template <typename R>
__global__ void __launch_bounds__(256)
	k_export(const typename CT<R>::T *__restrict__ d, uint64_t first,
		 uint64_t count, double2 *dst)
{
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
	     i += (uint64_t)gridDim.x * blockDim.x)
		dst[i] = to_c128(d[first + i]);
}

__global__ void k_copy_scal(const dk_scal *a, dk_scal *b) { *b = *a; }

/* Compare two registers of the same size (any precisions): per block
 * Re / Im of sum conj(x_i) y_i (scaled amplitudes) and max |x_i - y_i|. */
template <typename RA, typename RB>
__global__ void __launch_bounds__(256)
	k_compare(const typename CT<RA>::T *__restrict__ x, double sx,
		  const typename CT<RB>::T *__restrict__ y, double sy, uint64_t size,
		  double *partials)
{
	double re = 0.0, im = 0.0, mx = 0.0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
	     i += (uint64_t)gridDim.x * blockDim.x) {
		const double2 a = to_c128(__ldcs(x + i)), b = to_c128(__ldcs(y + i));
		const double ax = a.x * sx, ay = a.y * sx, bx = b.x * sy, by = b.y * sy;
		re += ax * bx + ay * by;
		im += ax * by - ay * bx;
		const double dx = ax - bx, dy = ay - by;
		mx = fmax(mx, sqrt(dx * dx + dy * dy));
	}
	block_sum2(re, im);
	__shared__ double red[32];
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
	if ((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = mx;
	__syncthreads();
	if (threadIdx.x == 0) {
		for (unsigned w = 1; w < (blockDim.x + 31) / 32; ++w)
			mx = fmax(mx, red[w]);
		partials[3 * blockIdx.x] = re;
		partials[3 * blockIdx.x + 1] = im;
		partials[3 * blockIdx.x + 2] = mx;
	}
}

__global__ void k_compare_finalize(const double *partials, int nb, double *out)
{
	if (threadIdx.x != 0)
		return;
	double re = 0.0, im = 0.0, mx = 0.0;
	for (int b = 0; b < nb; ++b) {
		re += partials[3 * b];
		im += partials[3 * b + 1];
		mx = fmax(mx, partials[3 * b + 2]);
	}
	out[0] = re;
	out[1] = im;
	out[2] = mx;
}

inline int grid_for(uint64_t work, int per_block, int cap)
{
	uint64_t b = (work + per_block - 1) / per_block;
	if (b < 1)
		b = 1;
	if (b > (uint64_t)cap)
		b = cap;
	return (int)b;
}

int g_num_sms = 148;

} // namespace

std::atomic<unsigned long long> g_launches{0};
int g_c64_tmem = 1;
int g_tm_allow_presplit = 1;
std::atomic<int> g_tm_ran{0};
std::atomic<unsigned long long> g_tm_presplit{0}, g_tm_entry_b{0};

/* ---------------------------------------------------------------------- */

/* Persistent sweeps walk tiles t = block, block + grid, ...  An in-place
 * sweep skips the tiles where its gates' conditions on qubits outside the
 * tile fail; such a condition is one bit of the tile number, so with an
 * even grid every block would see that bit fixed and half the blocks would
 * own all the work.  An odd grid makes each block's stride visit both
 * values of every tile-number bit. */
static uint64_t skip_balanced_grid(uint64_t blocks, const void *in, const void *out,
				   const dk_sweep_hdr *hp)
{
	if (in == out && !hp->all_touched && blocks > 1 && !(blocks & 1u))
		blocks--;
	return blocks;
}

template <typename R, int SW, int M, int MINB, int NBUF>
static cudaError_t run_sweep(const void *in, void *out, const unsigned char *dprog,
			     const dk_sweep_hdr *hp, int num_sms, const Scratch &s,
			     cudaStream_t st, int *blocks_out)
{
	typedef typename CT<R>::T C2;
	const int m = hp->m;
	const int nmat = (int)((hp->bytes - hp->mat_off) / 16);
	const size_t smem = NBUF * (sizeof(C2) << m) + (size_t)hp->ngate * sizeof(dk_gate_desc) +
			    (size_t)hp->ncond * sizeof(dk_gate_cond) + sizeof(C2) * (size_t)nmat;
	auto kern = k_sweep<R, SW, M, MINB, NBUF>;
	/* The limit is a per-function attribute shared by every thread: raise it
	 * once to the device maximum and never lower it, so concurrent launches
	 * of different sizes from different streams cannot race on it. */
	static std::once_flag once;
	static cudaError_t set_err = cudaSuccess;
	std::call_once(once, [&] {
		int dev = 0, maxopt = 0;
		cudaGetDevice(&dev);
		set_err = cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin,
						 dev);
		cudaFuncAttributes fa;
		if (set_err == cudaSuccess)
			set_err = cudaFuncGetAttributes(&fa, kern);
		/* the opt-in limit covers the kernel's static shared memory too */
		if (set_err == cudaSuccess)
			set_err = cudaFuncSetAttribute(kern,
						       cudaFuncAttributeMaxDynamicSharedMemorySize,
						       maxopt - (int)fa.sharedSizeBytes);
	});
	cudaError_t e = set_err;
	if (e != cudaSuccess)
		return e;
	uint64_t blocks = hp->ntiles;
	const uint64_t cap = (uint64_t)num_sms * MINB;
	if (blocks > cap)
		blocks = cap;
	blocks = skip_balanced_grid(blocks, in, out, hp);
	kern<<<(int)blocks, 1 << (m - DK_PASS_BITS), smem, st>>>((const C2 *)in, (C2 *)out,
								   dprog, s.partials);
	*blocks_out = (int)blocks;
	return cudaGetLastError();
}

template <typename R, int SW, int M, int MINB>
static cudaError_t run_sweep_tc(const void *in, void *out, const unsigned char *dprog,
				const dk_sweep_hdr *hp, int num_sms, const Scratch &s,
				cudaStream_t st, int *blocks_out)
{
	typedef typename CT<R>::T C2;
	const int m = hp->m;
	const size_t smem = (sizeof(C2) << m) + (size_t)hp->ngate * sizeof(dk_gate_desc) +
			    (size_t)hp->ncond * sizeof(dk_gate_cond);
	auto kern = k_sweep_tc<R, SW, M, MINB>;
	/* raised once to the device maximum, never lowered (see run_sweep) */
	static std::once_flag once;
	static cudaError_t set_err = cudaSuccess;
	std::call_once(once, [&] {
		int dev = 0, maxopt = 0;
		cudaGetDevice(&dev);
		set_err = cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin,
						 dev);
		cudaFuncAttributes fa;
		if (set_err == cudaSuccess)
			set_err = cudaFuncGetAttributes(&fa, kern);
		if (set_err == cudaSuccess)
			set_err = cudaFuncSetAttribute(kern,
						       cudaFuncAttributeMaxDynamicSharedMemorySize,
						       maxopt - (int)fa.sharedSizeBytes);
	});
	cudaError_t e = set_err;
	if (e != cudaSuccess)
		return e;
	uint64_t blocks = hp->ntiles;
	const uint64_t cap = (uint64_t)num_sms * MINB;
	if (blocks > cap)
		blocks = cap;
	blocks = skip_balanced_grid(blocks, in, out, hp);
	kern<<<(int)blocks, m >= 12 ? 256 : 1 << (m - DK_PASS_BITS), smem, st>>>((const C2 *)in, (C2 *)out,
								   dprog, s.partials);
	*blocks_out = (int)blocks;
	return cudaGetLastError();
}

/* Dynamic shared memory of a k_sweep_tm CTA: at least this much, so that no
 * SM holds more than two CTAs of it (or of any kernel with the same floor)
 * and their 2 x 256 tensor-memory columns always fit in the SM's 512. */
constexpr size_t kTmSmemFloor = 80u << 10;
/* and at most this much, so that two of them (with the kernel's static
 * shared memory) fit on an SM */
constexpr size_t kTmSmemMax = 106u << 10;

static cudaError_t run_sweep_tm(const void *in, void *out, const unsigned char *dprog,
				const dk_sweep_hdr *hp, int num_sms, const Scratch &s,
				cudaStream_t st, int *blocks_out)
{
	const size_t nmat = (hp->bytes - hp->mat_off) / 16; /* complex entries */
	const size_t mats_at = (2 * (sizeof(float2) << 12) + (size_t)hp->ngate * sizeof(dk_gate_desc) +
				(size_t)hp->ncond * sizeof(dk_gate_cond) +
				(size_t)hp->npass * sizeof(dk_pass_desc) + 1023) &
			       ~(size_t)1023;
	/* every matrix split once per CTA when they fit, else per entry */
	int pre = g_tm_allow_presplit;
	size_t smem = mats_at + (nmat / 64) * kTmBFloats * sizeof(float);
	if (!pre || smem > kTmSmemMax) {
		pre = 0;
		smem = mats_at + sizeof(float2) * nmat;
	}
	if (smem > kTmSmemMax)
		return cudaErrorNotSupported; /* the caller runs the sweep on mma.sync */
	if (smem < kTmSmemFloor)
		smem = kTmSmemFloor;
	auto kern = k_sweep_tm<4>;
	/* raised once to the device maximum, never lowered (see run_sweep) */
	static std::once_flag once;
	static cudaError_t set_err = cudaSuccess;
	std::call_once(once, [&] {
		int dev = 0, maxopt = 0;
		cudaGetDevice(&dev);
		set_err = cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin,
						 dev);
		cudaFuncAttributes fa;
		if (set_err == cudaSuccess)
			set_err = cudaFuncGetAttributes(&fa, kern);
		if (set_err == cudaSuccess)
			set_err = cudaFuncSetAttribute(kern,
						       cudaFuncAttributeMaxDynamicSharedMemorySize,
						       maxopt - (int)fa.sharedSizeBytes);
	});
	cudaError_t e = set_err;
	if (e != cudaSuccess)
		return e;
	uint64_t blocks = hp->ntiles;
	const uint64_t cap = (uint64_t)num_sms * 2;
	if (blocks > cap)
		blocks = cap;
	blocks = skip_balanced_grid(blocks, in, out, hp);
	kern<<<(int)blocks, 256, smem, st>>>((const float2 *)in, (float2 *)out, dprog,
					     s.partials, pre);
	*blocks_out = (int)blocks;
	g_tm_ran.store(1);
	(pre ? g_tm_presplit : g_tm_entry_b).fetch_add(1, std::memory_order_relaxed);
	return cudaGetLastError();
}

cudaError_t tm_fault_check(cudaStream_t st, unsigned *faults)
{
	*faults = 0;
	if (!g_tm_ran.load())
		return cudaSuccess;
	unsigned v = 0;
	cudaError_t e = cudaMemcpyFromSymbolAsync(&v, g_dk_tm_fault, sizeof(v), 0,
						  cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(st);
	if (e == cudaSuccess && v) {
		const unsigned zero = 0;
		e = cudaMemcpyToSymbolAsync(g_dk_tm_fault, &zero, sizeof(zero), 0,
					    cudaMemcpyHostToDevice, st);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(st);
	}
	*faults = v;
	return e;
}

cudaError_t launch_sweep(int prec, const void *in, void *out,
			 const unsigned char *dprog, const dk_sweep_hdr *hp,
			 const dk_scal *sc_in, dk_scal *sc_out, const Scratch &s,
			 int num_sms, cudaStream_t st)
{
	g_num_sms = num_sms;
	const int m = hp->m;
	int blocks = 0;
	cudaError_t e;
	if (hp->mode == DK_SWEEP_TENSOR && prec == DK_C64 && m == 12 && g_c64_tmem) {
		/* complex64, 12-bit tiles: tcgen05 TF32 products in tensor memory
		 * (a sweep whose tables exceed the kernel's shared memory runs on
		 * the mma.sync kernel below) */
		e = run_sweep_tm(in, out, dprog, hp, num_sms, s, st, &blocks);
		if (e == cudaErrorNotSupported)
			goto mma_sync;
		if (e != cudaSuccess)
			return e;
		const int all = hp->all_touched || (in != out);
		k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out, FIN_GATE, all);
		g_launches += 2;
		return cudaGetLastError();
	}
mma_sync:
	if (hp->mode == DK_SWEEP_TENSOR) {
		/* tensor-core passes (FP64 for complex128, split TF32 for
		 * complex64); tiles of 8 to 12 bits */
		if (prec == DK_C128)
			e = m >= 12 ? run_sweep_tc<double, 3, 12, DK_TC_MINB12>(in, out, dprog, hp,
										num_sms, s, st, &blocks)
				    : run_sweep_tc<double, 3, 11, DK_TC_MINB11>(in, out, dprog, hp,
										num_sms, s, st, &blocks);
		else
			e = m >= 12 ? run_sweep_tc<float, 4, 12, DK_TC_MINB12>(in, out, dprog, hp,
									       num_sms, s, st, &blocks)
				    : run_sweep_tc<float, 4, 11, DK_TC_MINB11>(in, out, dprog, hp,
									       num_sms, s, st, &blocks);
		if (e != cudaSuccess)
			return e;
		const int all = hp->all_touched || (in != out);
		k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out, FIN_GATE, all);
		g_launches += 2;
		return cudaGetLastError();
	}
	/* 12-bit tiles: one 512-thread CTA per SM, double-buffered; up to 11 bits:
	 * two 256-thread CTAs per SM, one buffer each */
	if (prec == DK_C128)
		e = m >= 12 ? run_sweep<double, 3, 12, 1, 2>(in, out, dprog, hp, num_sms, s, st,
							     &blocks)
			    : run_sweep<double, 3, 11, 2, 1>(in, out, dprog, hp, num_sms, s, st,
							     &blocks);
	else
		e = m >= 12 ? run_sweep<float, 4, 12, 1, 2>(in, out, dprog, hp, num_sms, s, st,
							    &blocks)
			    : run_sweep<float, 4, 11, 2, 1>(in, out, dprog, hp, num_sms, s, st,
							    &blocks);
	if (e != cudaSuccess)
		return e;
	const int all = hp->all_touched || (in != out);
	k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out, FIN_GATE, all);
	g_launches += 2;
	return cudaGetLastError();
}

cudaError_t launch_generic_gate(int prec, const void *in, void *out, unsigned n,
				unsigned k, const unsigned *tg, uint64_t cm,
				uint64_t am, const double *dmat,
				const dk_scal *sc_in, dk_scal *sc_out,
				const Scratch &s, cudaStream_t st)
{
	GenTargets t;
	for (unsigned j = 0; j < DK_MAX_GATE_QUBITS; ++j)
		t.t[j] = j < k ? (uint8_t)tg[j] : 0;
	const uint64_t size = 1ull << n;
	const int blocks = grid_for(size, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_generic<double><<<blocks, 256, 0, st>>>(
			(const double2 *)in, (double2 *)out, size, (int)k, t, cm, am,
			(const double2 *)dmat, s.partials);
	else
		k_generic<float><<<blocks, 256, 0, st>>>(
			(const float2 *)in, (float2 *)out, size, (int)k, t, cm, am,
			(const double2 *)dmat, s.partials);
	k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out, FIN_GATE, 1);
	g_launches += 2;
	return cudaGetLastError();
}

cudaError_t launch_init_zero(int prec, void *d, unsigned n, dk_scal *sc,
			     cudaStream_t st)
{
	const size_t bytes = (prec == DK_C128 ? 16 : 8) * ((size_t)1 << n);
	cudaError_t e = cudaMemsetAsync(d, 0, bytes, st);
	if (e != cudaSuccess)
		return e;
	if (prec == DK_C128)
		k_set_one<double><<<1, 1, 0, st>>>((double2 *)d, sc);
	else
		k_set_one<float><<<1, 1, 0, st>>>((float2 *)d, sc);
	g_launches += 1;
	return cudaGetLastError();
}

cudaError_t launch_import(int prec, const double *src, void *d, unsigned n,
			  dk_scal *sc, const Scratch &s, cudaStream_t st)
{
	const uint64_t size = 1ull << n;
	const int blocks = grid_for(size, 256 * 4, g_num_sms * 8);
	k_clear_flags<<<1, 1, 0, st>>>(sc);
	if (prec == DK_C128)
		k_import<double><<<blocks, 256, 0, st>>>((const double2 *)src,
							(double2 *)d, size, s.partials);
	else
		k_import<float><<<blocks, 256, 0, st>>>((const double2 *)src,
						       (float2 *)d, size, s.partials);
	k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc, sc, FIN_RESET, 1);
	g_launches += 3;
	return cudaGetLastError();
}

cudaError_t launch_read_half(int prec, const void *in, unsigned n, unsigned bit, int value,
			     double scale, void *dst, cudaStream_t st)
{
	const uint64_t half = 1ull << (n - 1);
	const int blocks = grid_for(half, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_read_half<double><<<blocks, 256, 0, st>>>((const double2 *)in, half, bit, value,
							    scale, (double2 *)dst);
	else
		k_read_half<float><<<blocks, 256, 0, st>>>((const float2 *)in, half, bit, value,
							   scale, (float2 *)dst);
	g_launches += 1;
	return cudaGetLastError();
}

cudaError_t launch_replace_half(int prec, const void *in, const void *src, unsigned n,
				unsigned bit, int value, double scale, void *out, dk_scal *sc,
				const Scratch &s, cudaStream_t st)
{
	const uint64_t size = 1ull << n;
	const int blocks = grid_for(size, 256 * 4, g_num_sms * 8);
	k_clear_flags<<<1, 1, 0, st>>>(sc);
	if (prec == DK_C128)
		k_replace_half<double><<<blocks, 256, 0, st>>>((const double2 *)in,
							       (const double2 *)src, size, bit,
							       value, scale, (double2 *)out,
							       s.partials);
	else
		k_replace_half<float><<<blocks, 256, 0, st>>>((const float2 *)in, (const float2 *)src,
							      size, bit, value, scale, (float2 *)out,
							      s.partials);
	k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc, sc, FIN_RESET, 1);
	g_launches += 3;
	return cudaGetLastError();
}

/* k_marginals with the smallest accumulator array that holds the n - sbits
 * bits each thread varies over. */
static void launch_marginals_kernel(int prec, const void *d, unsigned n, int sbits, int blocks,
				    int threads, double *partials, cudaStream_t st)
{
	const int nb = (int)n - sbits;
#define DK_MARG(NB)                                                                      \
	do {                                                                             \
		if (prec == DK_C128)                                                     \
			k_marginals<double, NB><<<blocks, threads, 0, st>>>(             \
				(const double2 *)d, (int)n, sbits, partials);            \
		else                                                                     \
			k_marginals<float, NB><<<blocks, threads, 0, st>>>(              \
				(const float2 *)d, (int)n, sbits, partials);             \
	} while (0)
	if (nb <= 12)
		DK_MARG(12);
	else if (nb <= 16)
		DK_MARG(16);
	else
		DK_MARG(kMargHi);
#undef DK_MARG
}

cudaError_t launch_marginals(int prec, const void *d, unsigned n, const Scratch &s,
			     cudaStream_t st)
{
	/* up to 2048 blocks: 2 per SM make 6.9 waves of 296 at 30 qubits */
	int threads = 256, blocks = 1;
	if (n < 8)
		threads = 1 << n;
	else {
		int lb = (int)n - 8;
		if (lb > 11)
			lb = 11;
		blocks = 1 << lb;
	}
	int sbits = 0;
	while ((1 << sbits) < threads * blocks)
		sbits++;
	if ((int)n - sbits > kMargHi)
		return cudaErrorInvalidValue;
	if (threads < 32) {
		/* tiny registers: one warp, lanes beyond the register are idle */
		threads = 32;
		sbits = (int)n;
	}
	launch_marginals_kernel(prec, d, n, sbits, blocks, threads, s.partials, st);
	k_marg_finalize<<<1, 64, 0, st>>>(s.partials, blocks, (int)n, s.marg);
	g_launches += 2;
	return cudaGetLastError();
}

cudaError_t launch_marginals_blocks(int prec, const void *d, unsigned n,
				    const Scratch &s, int max_blocks, cudaStream_t st)
{
	int threads = 256, blocks = 1;
	if (n < 8)
		threads = 1 << n;
	else {
		int lb = (int)n - 8;
		while (lb > 0 && (1 << lb) > max_blocks)
			lb--;
		blocks = 1 << lb;
	}
	int sbits = 0;
	while ((1 << sbits) < threads * blocks)
		sbits++;
	if ((int)n - sbits > kMargHi)
		return cudaErrorInvalidValue;
	if (threads < 32) {
		threads = 32;
		sbits = (int)n;
	}
	/* cudaLaunchKernel returns the status of this launch alone: an error
	 * left pending by the caller's earlier, unrelated work is neither
	 * reported as this call's failure nor cleared */
	const int nb = (int)n - sbits;
	const void *kern;
	if (prec == DK_C128)
		kern = nb <= 12 ? (const void *)k_marginals<double, 12>
		       : nb <= 16 ? (const void *)k_marginals<double, 16>
				  : (const void *)k_marginals<double, kMargHi>;
	else
		kern = nb <= 12 ? (const void *)k_marginals<float, 12>
		       : nb <= 16 ? (const void *)k_marginals<float, 16>
				  : (const void *)k_marginals<float, kMargHi>;
	const void *amps = d;
	int ni = (int)n, sb = sbits;
	double *partials = s.partials, *marg = s.marg;
	void *kargs[] = { (void *)&amps, (void *)&ni, (void *)&sb, (void *)&partials };
	cudaError_t e = cudaLaunchKernel(kern, dim3(blocks), dim3(threads), kargs, 0, st);
	if (e != cudaSuccess)
		return e;
	int nblk = blocks;
	void *fargs[] = { (void *)&partials, (void *)&nblk, (void *)&ni, (void *)&marg };
	e = cudaLaunchKernel((const void *)k_marg_finalize, dim3(1), dim3(64), fargs, 0, st);
	g_launches += (e == cudaSuccess) ? 2 : 1;
	return e;
}

cudaError_t launch_measure_collapse(int prec, const void *in, void *out,
				    unsigned n, unsigned q, double roll,
				    int forced, const dk_scal *sc_in,
				    dk_scal *sc_out, const Scratch &s,
				    cudaStream_t st)
{
	k_decide<<<1, 1, 0, st>>>(s.marg, (int)q, roll, forced, sc_in, sc_out);
	const uint64_t half = 1ull << (n - 1);
	if (out != nullptr) {
		const int blocks = grid_for(half, 256 * 4, g_num_sms * 8);
		if (prec == DK_C128)
			k_collapse<double><<<blocks, 256, 0, st>>>(
				(const double2 *)in, (double2 *)out, half, (int)q,
				sc_out, s.partials);
		else
			k_collapse<float><<<blocks, 256, 0, st>>>(
				(const float2 *)in, (float2 *)out, half, (int)q,
				sc_out, s.partials);
		k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out,
					       FIN_COLLAPSE, 1);
	}
	g_launches += (out != nullptr) ? 3 : 1;
	return cudaGetLastError();
}

cudaError_t launch_measure_joint(int prec, const void *in, void *out, unsigned n,
				 uint64_t mask, const double *rolls_dev, int32_t *flags_dev,
				 const dk_scal *sc_in, dk_scal *sc_out, const Scratch &s,
				 cudaStream_t st)
{
	const int k = __builtin_popcountll(mask);
	if (k < 1 || k > kJointMaxQubits || (unsigned)k > n)
		return cudaErrorInvalidValue;
	DepRuns runs;
	memset(&runs, 0, sizeof(runs));
	unsigned src = 0;
	for (unsigned q = 0; q < n;) {
		if ((mask >> q) & 1u) {
			++q;
			continue;
		}
		unsigned e = q;
		while (e < n && !((mask >> e) & 1u))
			++e;
		runs.src[runs.nruns] = (uint8_t)src;
		runs.dst[runs.nruns] = (uint8_t)q;
		runs.len[runs.nruns] = (uint8_t)(e - q);
		runs.nruns++;
		src += e - q;
		q = e;
	}
	const uint64_t nbins = 1ull << k, per_bin = 1ull << (n - k);
	/* chunks of >= 4096 amplitudes, at most kJointPartials partials */
	uint64_t nchunk = (per_bin + 4095) / 4096;
	if (nchunk * nbins > kJointPartials)
		nchunk = kJointPartials / nbins;
	if (nchunk < 1)
		nchunk = 1;
	const uint64_t chunk = (per_bin + nchunk - 1) / nchunk;
	double *part = s.partials;
	double *joint = s.partials + kJointPartials;
	uint64_t *vbits = reinterpret_cast<uint64_t *>(s.u64 + 1);
	if (k <= 4 && n >= 12) {
		/* one contiguous pass, 2048 blocks at most */
		uint32_t qpack = 0;
		int j = 0;
		for (unsigned q = 0; q < n; ++q)
			if ((mask >> q) & 1u)
				qpack |= q << (8 * j++);
		const uint64_t size = 1ull << n;
		uint64_t nb = size / kJointSeg;
		if (nb > 2048)
			nb = 2048;
		if (prec == DK_C128)
			k_joint_small<double><<<(unsigned)nb, 256, 0, st>>>((const double2 *)in, size,
									    qpack, k, part);
		else
			k_joint_small<float><<<(unsigned)nb, 256, 0, st>>>((const float2 *)in, size,
									   qpack, k, part);
		k_joint_finalize<<<(unsigned)nbins, 256, 0, st>>>(part, nb, joint);
	} else {
		uint64_t gx = nchunk < (uint64_t)g_num_sms * 8 ? nchunk : (uint64_t)g_num_sms * 8;
		dim3 grid((unsigned)gx, (unsigned)nbins);
		if (prec == DK_C128)
			k_joint<double><<<grid, 256, 0, st>>>((const double2 *)in, runs, mask,
							      per_bin, chunk, nchunk, part);
		else
			k_joint<float><<<grid, 256, 0, st>>>((const float2 *)in, runs, mask,
							     per_bin, chunk, nchunk, part);
		k_joint_finalize<<<(unsigned)nbins, 256, 0, st>>>(part, nchunk, joint);
	}
	k_decide_joint<<<1, 32, 0, st>>>(joint, k, rolls_dev, flags_dev, vbits, mask, sc_in, sc_out);
	g_launches += 3;
	if (out != nullptr) {
		const int blocks = grid_for(per_bin, 256 * 4, g_num_sms * 8);
		if (prec == DK_C128)
			k_collapse_joint<double><<<blocks, 256, 0, st>>>(
				(const double2 *)in, (double2 *)out, runs, per_bin, vbits, s.partials,
				1ull << n);
		else
			k_collapse_joint<float><<<blocks, 256, 0, st>>>(
				(const float2 *)in, (float2 *)out, runs, per_bin, vbits, s.partials,
				1ull << n);
		k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_in, sc_out, FIN_COLLAPSE, 1);
		g_launches += 2;
	}
	return cudaGetLastError();
}

cudaError_t launch_join(int prec, const void *most, unsigned n1,
			const dk_scal *sc1, const void *least, unsigned n2,
			const dk_scal *sc2, void *out, dk_scal *sc_out,
			const Scratch &s, cudaStream_t st)
{
	const uint64_t size = 1ull << (n1 + n2);
	k_clear_flags<<<1, 1, 0, st>>>(sc_out);
	const size_t least_bytes = (prec == DK_C128 ? 16ull : 8ull) << n2;
	if (least_bytes > (32ull << 20) && n1 <= 10) {
		/* least does not stay in the L2 across most amplitudes */
		const int wb = grid_for(1ull << n2, 256 * 4, g_num_sms * 8);
		if (prec == DK_C128)
			k_join_wide<double><<<wb, 256, 0, st>>>((const double2 *)most, sc1,
								(const double2 *)least, sc2, (int)n1,
								(int)n2, (double2 *)out, s.partials);
		else
			k_join_wide<float><<<wb, 256, 0, st>>>((const float2 *)most, sc1,
							       (const float2 *)least, sc2, (int)n1,
							       (int)n2, (float2 *)out, s.partials);
		k_finalize<<<1, 256, 0, st>>>(s.partials, wb, sc_out, sc_out, FIN_RESET, 1);
		g_launches += 3;
		return cudaGetLastError();
	}
	const int blocks = grid_for(size, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_join<double><<<blocks, 256, 0, st>>>((const double2 *)most, sc1,
						      (const double2 *)least, sc2,
						      (int)n2, (double2 *)out, size,
						      s.partials);
	else
		k_join<float><<<blocks, 256, 0, st>>>((const float2 *)most, sc1,
						     (const float2 *)least, sc2, (int)n2,
						     (float2 *)out, size, s.partials);
	k_finalize<<<1, 256, 0, st>>>(s.partials, blocks, sc_out, sc_out, FIN_RESET, 1);
	g_launches += 3;
	return cudaGetLastError();
}

cudaError_t launch_first_nonzero(int prec, const void *d, uint64_t first,
				 uint64_t count, const Scratch &s, cudaStream_t st)
{
	cudaError_t e = cudaMemsetAsync(s.u64, 0xff, sizeof(unsigned long long), st);
	if (e != cudaSuccess)
		return e;
	const int blocks = grid_for(count, 256, g_num_sms * 8);
	if (prec == DK_C128)
		k_first_nz<double><<<blocks, 256, 0, st>>>((const double2 *)d, first,
							  count, s.u64);
	else
		k_first_nz<float><<<blocks, 256, 0, st>>>((const float2 *)d, first,
							 count, s.u64);
	g_launches += 1;
	return cudaGetLastError();
}

cudaError_t launch_gather_kept(int prec, const void *d, unsigned n,
			       uint64_t keep_mask, double2 *M, cudaStream_t st)
{
	const uint64_t full = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
	const uint64_t trace = full & ~keep_mask;
	const int k = __builtin_popcountll(keep_mask);
	const uint64_t total = 1ull << n;
	if (prec == DK_C64 && keep_mask == (1ull << k) - 1ull && n >= 1) {
		const uint64_t pairs = total >> 1;
		k_widen_c64<<<grid_for(pairs, 256 * 4, g_num_sms * 8), 256, 0, st>>>(
			(const float4 *)d, (double4 *)M, pairs);
		g_launches += 1;
		return cudaGetLastError();
	}
	const int blocks = grid_for(total, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_gather_kept<double><<<blocks, 256, 0, st>>>((const double2 *)d,
							     keep_mask, trace, k,
							     total, M);
	else
		k_gather_kept<float><<<blocks, 256, 0, st>>>((const float2 *)d,
							    keep_mask, trace, k, total,
							    M);
	g_launches += 1;
	return cudaGetLastError();
}

cudaError_t launch_herm_fill(const double2 *C, double2 *rho, uint64_t dim,
			     cudaStream_t st)
{
	const int blocks = grid_for(dim * dim, 256 * 4, g_num_sms * 8);
	k_herm_fill<<<blocks, 256, 0, st>>>(C, rho, dim);
	g_launches += 1;
	return cudaGetLastError();
}

/* Dynamic shared memory of k_rho_tc: two slab buffers of the row and column
 * tiles.  The attribute is set once; the occupancy it allows is cached. */
constexpr size_t kRhoSmem = sizeof(double2) * 2 * 2 * kRhoSlab * kRhoTile;

static cudaError_t rho_prepare(int *ctas_per_sm)
{
	static std::once_flag once;
	static cudaError_t err = cudaSuccess;
	static int occ = 1;
	std::call_once(once, [&] {
		err = cudaFuncSetAttribute(k_rho_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
					   (int)kRhoSmem);
		int o = 0;
		if (err == cudaSuccess &&
		    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_rho_tc, 256, kRhoSmem) ==
			    cudaSuccess &&
		    o > 0)
			occ = o;
		cudaGetLastError();
	});
	if (ctas_per_sm)
		*ctas_per_sm = occ;
	return err;
}

/* Traced-range splits of the reduced density product.  Tiles x splits CTAs
 * should fill whole waves of the resident CTA slots (a 1024 x 1024 result
 * has 136 tiles; 13 splits fill 12 waves of 148 at 99.5 %, where 8 would
 * leave the last of 8 waves a third full); each split keeps at least 256
 * traced values, there are at most 64 and their partials stay within 1 GiB.
 * Among split counts giving at least two waves, a larger count is taken only
 * when it fills the waves 2 % better. */
int rho_splits(uint64_t dim, uint64_t K, int num_sms)
{
	if (dim < (uint64_t)kRhoTile) {
		uint64_t ns = (K + 4095) / 4096; /* traced values per small CTA: 4096 */
		if (ns > 1024)
			ns = 1024;
		return ns ? (int)ns : 1;
	}
	const uint64_t T = dim / kRhoTile, ntile = T * (T + 1) / 2;
	int occ = 1;
	rho_prepare(&occ);
	const uint64_t slots = (uint64_t)(num_sms > 0 ? num_sms : 1) * (uint64_t)occ;
	const uint64_t part_cap = (1ull << 30) / (16 * dim * dim);
	uint64_t best = 1;
	double best_fill = -1.0;
	for (uint64_t ns = 1; ns <= 64 && ns * 256 <= K && (ns == 1 || ns <= part_cap); ++ns) {
		const uint64_t ctas = ntile * ns;
		const bool more_allowed = ns < 64 && (ns + 1) * 256 <= K && ns + 1 <= part_cap;
		if (ctas < 2 * slots && more_allowed)
			continue;
		const uint64_t waves = (ctas + slots - 1) / slots;
		const double fill = (double)ctas / (double)(waves * slots);
		if (fill > best_fill + 0.02) {
			best = ns;
			best_fill = fill;
		}
	}
	return (int)best;
}

cudaError_t launch_rho(const double2 *A, uint64_t dim, uint64_t K, double alpha, int nsplit,
		       double2 *part, double2 *C, cudaStream_t st)
{
	if (dim < (uint64_t)kRhoTile) {
		const uint64_t bchunk = (K + nsplit - 1) / nsplit;
		k_rho_small<<<nsplit, 256, 0, st>>>(A, (uint32_t)dim, K, bchunk, part);
		const int blocks = grid_for(dim * dim, 256, g_num_sms * 8);
		k_rho_reduce<<<blocks, 256, 0, st>>>(part, nsplit, dim, alpha, C);
		g_launches += 2;
		return cudaGetLastError();
	}
	const uint64_t T = dim / kRhoTile, ntile = T * (T + 1) / 2;
	uint64_t bchunk = (K + nsplit - 1) / nsplit;
	bchunk = (bchunk + kRhoSlab - 1) / kRhoSlab * kRhoSlab;
	const cudaError_t set_err = rho_prepare(nullptr);
	if (set_err != cudaSuccess)
		return set_err;
	dim3 grid((unsigned)ntile, (unsigned)nsplit);
	k_rho_tc<<<grid, 256, kRhoSmem, st>>>(A, dim, K, bchunk, nsplit == 1 ? C : part, alpha);
	g_launches += 1;
	if (nsplit > 1) {
		const int blocks = grid_for(dim * dim, 256 * 4, g_num_sms * 8);
		k_rho_reduce<<<blocks, 256, 0, st>>>(part, nsplit, dim, alpha, C);
		g_launches += 1;
	}
	return cudaGetLastError();
}

cudaError_t launch_rho_elem(int prec, const void *d, unsigned n,
			    uint64_t keep_mask, uint64_t i, uint64_t j,
			    const dk_scal *sc, const Scratch &s, cudaStream_t st)
{
	const uint64_t full = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
	const uint64_t trace = full & ~keep_mask;
	const int t = __builtin_popcountll(trace);
	/* host-side deposit of the kept indices */
	uint64_t ia = 0, ib = 0, m = keep_mask;
	for (uint64_t bit = 1; m; bit <<= 1) {
		const uint64_t low = m & (~m + 1ull);
		if (i & bit)
			ia |= low;
		if (j & bit)
			ib |= low;
		m &= m - 1ull;
	}
	const uint64_t cnt = 1ull << t;
	const int blocks = grid_for(cnt, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_rho_elem<double><<<blocks, 256, 0, st>>>((const double2 *)d, ia, ib,
							  trace, cnt, s.partials);
	else
		k_rho_elem<float><<<blocks, 256, 0, st>>>((const float2 *)d, ia, ib,
							 trace, cnt, s.partials);
	k_rho_elem_finalize<<<1, 32, 0, st>>>(s.partials, blocks, sc, s.marg);
	g_launches += 2;
	return cudaGetLastError();
}

cudaError_t launch_export(int prec, const void *d, uint64_t first, uint64_t count,
			  double2 *dst, cudaStream_t st)
{
	const int blocks = grid_for(count, 256 * 4, g_num_sms * 8);
	if (prec == DK_C128)
		k_export<double><<<blocks, 256, 0, st>>>((const double2 *)d, first,
							count, dst);
	else
		k_export<float><<<blocks, 256, 0, st>>>((const float2 *)d, first, count,
						       dst);
	g_launches += 1;
	return cudaGetLastError();
}

cudaError_t launch_compare(int prec_x, const void *x, double sx, int prec_y, const void *y,
			   double sy, unsigned n, const Scratch &s, cudaStream_t st)
{
	const uint64_t size = 1ull << n;
	const int blocks = grid_for(size, 256 * 4, g_num_sms * 8);
	if (prec_x == DK_C128 && prec_y == DK_C128)
		k_compare<double, double><<<blocks, 256, 0, st>>>((const double2 *)x, sx,
								  (const double2 *)y, sy, size,
								  s.partials);
	else if (prec_x == DK_C64 && prec_y == DK_C128)
		k_compare<float, double><<<blocks, 256, 0, st>>>((const float2 *)x, sx,
								 (const double2 *)y, sy, size,
								 s.partials);
	else if (prec_x == DK_C128 && prec_y == DK_C64)
		k_compare<double, float><<<blocks, 256, 0, st>>>((const double2 *)x, sx,
								 (const float2 *)y, sy, size,
								 s.partials);
	else
		k_compare<float, float><<<blocks, 256, 0, st>>>((const float2 *)x, sx,
								(const float2 *)y, sy, size,
								s.partials);
	k_compare_finalize<<<1, 32, 0, st>>>(s.partials, blocks, s.marg);
	g_launches += 2;
	return cudaGetLastError();
}

cudaError_t launch_copy(int prec, const void *src, void *dst, unsigned n,
			const dk_scal *sc_in, dk_scal *sc_out, cudaStream_t st)
{
	const size_t bytes = (prec == DK_C128 ? 16 : 8) * ((size_t)1 << n);
	cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
	if (e != cudaSuccess)
		return e;
	k_copy_scal<<<1, 1, 0, st>>>(sc_in, sc_out);
	g_launches += 1;
	return cudaGetLastError();
}

} // namespace dk

#ifdef DK_DEBUG_CHECKS
/* Debug builds only: the first failed index check since the last reset, or 0
 * (site in bits 56-63, index in bits 0-55); `reset` clears the record.  Call
 * dk_sync() first so that every kernel has finished. */
extern "C" int dk_debug_checks(uint64_t *first_failure, int reset)
{
	unsigned long long v = 0;
	if (cudaMemcpyFromSymbol(&v, dk::g_dk_check, sizeof(v)) != cudaSuccess) {
		cudaGetLastError();
		return DK_ERR_CUDA;
	}
	if (reset) {
		const unsigned long long zero = 0;
		if (cudaMemcpyToSymbol(dk::g_dk_check, &zero, sizeof(zero)) != cudaSuccess) {
			cudaGetLastError();
			return DK_ERR_CUDA;
		}
	}
	if (first_failure)
		*first_failure = v;
	return DK_OK;
}

/* Debug builds only: 1 makes every later tcgen05 sweep wait on an mbarrier
 * that nothing arrives at (its bounded waits expire and the next read of
 * the register returns DK_ERR_TIMEOUT); 0 restores normal operation. */
extern "C" int dk_debug_tm_starve(int on)
{
	const int v = on ? 1 : 0;
	if (cudaMemcpyToSymbol(dk::g_dk_tm_starve, &v, sizeof(v)) != cudaSuccess) {
		cudaGetLastError();
		return DK_ERR_CUDA;
	}
	return DK_OK;
}
#endif
