// Fifth-generation tensor core (tcgen05) building blocks for sm_100a, in
// inline PTX: shared-memory matrix descriptors, the kind::f16 MMA with its
// accumulator in tensor memory (TMEM), commits to an mbarrier, TMEM
// allocation and loads.
//
// Operand layout used throughout (no swizzle): a tile of R rows x K columns
// of 16-bit elements is stored as 8x8 "core matrices" of 128 contiguous bytes
// (8 rows of 16 bytes), core matrix (r / 8, k / 8) at byte
//     (r / 8) * (K / 8) * 128 + (k / 8) * 128,
// element (r % 8, k % 8) at 16 * (r % 8) + 2 * (k % 8) inside it. Read with
// K as the reduction dimension ("K-major") the descriptor's leading byte
// offset is 128 (the next 8 columns) and its stride byte offset
// (K / 8) * 128 (the next 8 rows). The same bytes read with the rows as the
// reduction dimension ("MN-major", the transpose) have stride byte offset 128
// (the next 8 columns) and leading byte offset (K / 8) * 128.
#pragma once

#include <cstdint>

namespace restir
{
namespace umma
{

__device__ __forceinline__ uint32_t smemAddress(const void* p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in a tile with k columns (a multiple of 8).
__host__ __device__ __forceinline__ uint32_t coreOffset(uint32_t r, uint32_t k, uint32_t columns)
{
	return (r >> 3) * (columns >> 3) * 128u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t smemDescriptor(uint32_t address, uint32_t leadingBytes, uint32_t strideBytes)
{
	uint64_t d = 0;
	d |= uint64_t((address >> 4) & 0x3fffu);
	d |= uint64_t((leadingBytes >> 4) & 0x3fffu) << 16;
	d |= uint64_t((strideBytes >> 4) & 0x3fffu) << 32;
	d |= uint64_t(1) << 46;
	return d;
}

// Instruction descriptor of kind::f16: bfloat16 A and B, FP32 accumulator,
// M x N, each operand K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t instrDescriptorBf16(uint32_t m, uint32_t n, uint32_t aMajor, uint32_t bMajor)
{
	return (1u << 4)           // D: F32
		| (1u << 7)            // A: BF16
		| (1u << 10)           // B: BF16
		| (aMajor << 15)
		| (bMajor << 16)
		| ((n >> 3) << 17)
		| ((m >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 step; issued by one thread.
__device__ __forceinline__ void mma(uint32_t tmemD, uint64_t aDescriptor, uint64_t bDescriptor, uint32_t instr,
	bool accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
		:
		: "r"(tmemD), "l"(aDescriptor), "l"(bDescriptor), "r"(instr), "r"(uint32_t(accumulate))
		: "memory");
}

// Arrives on the mbarrier when every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint32_t barrier)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(barrier) : "memory");
}

__device__ __forceinline__ void barrierInit(uint32_t barrier, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(barrier), "r"(count) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the barrier's phase with this parity; gives up after `limit`
// polls (each poll itself waits a little) and returns false.
__device__ __forceinline__ bool barrierWait(uint32_t barrier, uint32_t parity, uint32_t limit)
{
	for (uint32_t i = 0; i < limit; ++i)
	{
		uint32_t done = 0;
		asm volatile(
			"{\n\t.reg .pred p;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, p;\n\t}\n"
			: "=r"(done)
			: "r"(barrier), "r"(parity)
			: "memory");
		if (done != 0u)
		{
			return true;
		}
	}
	return false;
}

// TMEM allocation by one whole warp; the base address lands in *slot.
__device__ __forceinline__ void tmemAllocate(uint32_t slot, uint32_t columns)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(columns) : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemFree(uint32_t base, uint32_t columns)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync()
{
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fenceAfterSync()
{
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Makes this thread's shared-memory stores visible to the tensor cores.
__device__ __forceinline__ void fenceSharedForAsync()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 consecutive 32-bit columns of this warp's 32 TMEM lanes (lane = thread);
// address = base + (first lane << 16) + first column.
__device__ __forceinline__ void tmemLoad16(uint32_t address, float* v)
{
	uint32_t r[16];
	// The load and its wait in one statement: the registers are defined only
	// after the wait.
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 "
		"{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
		"tcgen05.wait::ld.sync.aligned;"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(address)
		: "memory");
#pragma unroll
	for (int i = 0; i < 16; ++i)
	{
		v[i] = __uint_as_float(r[i]);
	}
}

} // namespace umma
} // namespace restir
