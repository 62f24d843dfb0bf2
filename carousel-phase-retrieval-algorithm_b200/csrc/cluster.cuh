// Thread-block clusters: a pattern spread over the shared memory of several
// CTAs (distributed shared memory, one SM each).
//
// A CTA reaches another CTA's shared memory of the same cluster through the
// shared::cluster window: mapa turns an address of this CTA's shared memory
// into the address of the same variable in the CTA of a given rank.  The
// kernels here only ever write remote shared memory, never read it: bulk
// copies of blocks of their own shared memory (below), and single stores
// (st.shared::cluster) ordered by a cluster barrier (arrive with release, wait
// with acquire, both at cluster scope).  All threads of all CTAs of the
// cluster take part in each barrier; the hardware barrier needs no spinning
// code of its own.
//
// Before the first remote write every CTA of the cluster must be running,
// and no CTA may exit while another can still write into its shared memory
// or a copy can still read its own: a kernel therefore passes one cluster
// barrier before its first remote write and one after its last.
#pragma once
#include <cstdint>

#include "cpra_common.cuh"

namespace cpra_b200 {

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// the shared::cluster address of `local` (a shared::cta address of this CTA)
// in the CTA of rank `rank`
__device__ __forceinline__ uint32_t cluster_map(uint32_t local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_store(uint32_t addr, Cx<float> v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void cluster_store(uint32_t addr, float v) {
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

// every thread of every CTA of the cluster: remote stores before it are
// visible to all accesses after it
__device__ __forceinline__ void cluster_sync() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::
            : "memory");
}

// ---- block transfers between the CTAs' shared memories, counted on mbarriers ----
//
// A CTA moves a contiguous block of its own shared memory into another CTA's
// with one bulk copy (the SM's copy engine; no registers held, no fence on
// the issuing threads).  The copy completes its byte count as transactions
// on an mbarrier in the receiving CTA; the receiver arms the barrier with the
// bytes it expects in a phase and waits for the phase to complete, after
// which the data is visible to its threads.  Shared memory written by the
// threads and then read by a copy (or written by the threads after a copy
// wrote it) needs fence.proxy.async between the two: the copies run in the
// async proxy.

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(arrivals) : "memory");
}
// barrier initialisations of this thread visible to the cluster's copies
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// the thread's arrival, expecting `bytes` more of transactions in the current phase
__device__ __forceinline__ void mbar_arrive_expect(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of parity `parity` to complete, at most `limit_ns`
// nanoseconds; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_test(mbar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_test(mbar, parity))
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}

// this thread's generic-proxy shared-memory accesses ordered before later
// async-proxy (copy) accesses
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// `bytes` (a multiple of 16; both addresses 16-byte aligned) from this CTA's
// shared memory at src to the shared::cluster address dst, completing `bytes`
// transactions on the mbarrier at the shared::cluster address mbar (in the
// CTA that owns dst)
__device__ __forceinline__ void bulk_copy_to_cta(uint32_t dst, uint32_t src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst),
                 "r"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

}  // namespace cpra_b200
