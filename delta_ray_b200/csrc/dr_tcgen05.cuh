// Blackwell (sm_100a) tensor-core primitives in inline PTX: shared-memory
// matrix descriptors, the tcgen05 instruction descriptor, tcgen05.mma with
// TMEM accumulators, tcgen05.commit to an mbarrier, TMEM allocation and loads.
//
// Operands live in shared memory in the no-swizzle interleaved layout: 8 x 8
// bf16 "core matrices" of 128 contiguous bytes (8 rows of 16 bytes).  For a
// matrix of R rows whose C columns are the contiguous dimension,
//   byte offset (r, c) = ((r / 8) * (C / 8) + c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2.
// Read as a K-major operand (rows = M or N, columns = K) its descriptor has
// LBO = 128 (next 8 columns) and SBO = C / 8 * 128 (next 8 rows); read as an
// MN-major operand (columns = M or N, rows = K) the same bytes have SBO = 128
// (next 8 columns) and LBO = C / 8 * 128 (next 8 rows).  One buffer therefore
// serves as A of a forward product and as the transposed operand of the
// weight-gradient product.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#define TC_DEV static __device__ __forceinline__

namespace tc {

TC_DEV uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__host__ __device__ constexpr uint32_t imat_offset(int r, int c, int C) {
    return (uint32_t)((((r >> 3) * (C >> 3) + (c >> 3)) << 7) + ((r & 7) << 4) + ((c & 7) << 1));
}

// Shared-memory matrix descriptor (no swizzle, version 1 for sm_100).
TC_DEV uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major view of an interleaved matrix with C contiguous columns.
TC_DEV uint64_t sdesc_k(uint32_t addr, int C) { return sdesc(addr, 128u, (uint32_t)(C >> 3) << 7); }
// MN-major view of the same matrix.
TC_DEV uint64_t sdesc_mn(uint32_t addr, int C) { return sdesc(addr, (uint32_t)(C >> 3) << 7, 128u); }

// Instruction descriptor of kind::f16: bf16 A and B, f32 accumulator,
// M x N tile, A / B K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread.
TC_DEV void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// Arrive on the mbarrier once every tcgen05.mma issued so far by this thread completed.
TC_DEV void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

TC_DEV void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the mbarrier phase `parity` to complete; gives up after `limit`
// polls (each poll may suspend the thread for a while) and returns false.
TC_DEV bool mbar_wait(uint32_t mbar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

TC_DEV void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
TC_DEV void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
TC_DEV void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole warp;
// the base address is written to shared memory at `slot`.
TC_DEV void tmem_alloc(uint32_t slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
TC_DEV void tmem_free(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// 32 consecutive f32 columns of this thread's TMEM lane (32x32b shape: warp w
// reads lanes 32w..32w+31).  Complete with ld_wait() before using v.
TC_DEV void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Writes 8 bf16 values (16 bytes) of row r, columns c0..c0+7 (c0 % 8 == 0), of
// an interleaved matrix with C columns.
TC_DEV void st_row8(uint8_t *base, int r, int c0, int C, const float *v) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4 *>(base + imat_offset(r, c0, C)) = *reinterpret_cast<uint4 *>(h);
}
TC_DEV void ld_row8(const uint8_t *base, int r, int c0, int C, float *v) {
    uint4 u = *reinterpret_cast<const uint4 *>(base + imat_offset(r, c0, C));
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

}  // namespace tc
