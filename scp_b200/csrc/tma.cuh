// tma.cuh -- plane staging of the FP64 fused step through the Tensor Memory
// Accelerator.
//
// A plane of the CTA's column is the (TY + 2) x TX block of every field (the
// tile's rows plus one halo row on either side in j) and two halo columns in
// k.  One tiled TMA load per field moves the block: a 4-D tensor map over the
// position buffer, dimensions (k, j, i, field), box TX x rows x 1 x 1.  The
// periodic wrap in j is a second pair of boxes for the tiles on the j edges
// (TY + 1 rows from the tile, plus the wrapped row); the two halo columns
// (k0 - 1 and k0 + TX, wrapped; 2 TY values per field, plus the two corners the
// gauged plaquettes read) are single doubles copied by the CTA's threads with
// cp.async, one or two per thread.  Each ring slot has an mbarrier that the
// block loads complete with their byte count; every wait on it is bounded.
//
// Requirements (checked on the host): FP64, N a multiple of TX and of TY,
// N >= 2 TY, N even (16-byte row pitch); every tensor map covers the
// handle's own position buffer on this GPU, and no load multicasts.
#pragma once
#include <cuda.h>

#include "step.cuh"

namespace scp {

// The three tensor maps of one position buffer: TY + 2 rows (interior tiles),
// TY + 1 rows and one row (tiles on the j edges).
struct TmaMaps {
    CUtensorMap full, part, row;
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// tiled 4-D load of one box into shared memory, completing on bar
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

constexpr unsigned kTmaWaitLimit = 1u << 24;   // try_wait rounds before a wait gives up
constexpr int kFlagTimeout = 2;                 // bit of the handle's flag word: a bounded wait gave up

// Ring depth of the TMA staging: planes i, i+1 resident and i+2, i+3 in flight
// (a deeper ring costs shared memory only, no registers).
constexpr int kTmaSlots = 4;

template <int TX, int TY, bool GAUGED>
struct TmaLayout {
    static constexpr int NF = GAUGED ? 15 : 12;
    static constexpr int ROWS = TY + 2;
    static constexpr int MAIN = ROWS * TX;                       // block of one field
    static constexpr int LEFT = MAIN, RIGHT = MAIN + ROWS;       // halo columns k0 - 1, k0 + TX
    static constexpr int FS = (MAIN + 2 * ROWS + 15) / 16 * 16;  // field stride: 128-byte aligned blocks
    static constexpr int SLOT = NF * FS;
    static constexpr int NT = TX * TY;
    static constexpr int NHALO = 2 * TY * NF + (GAUGED ? 6 : 0); // halo-column doubles per plane
    static constexpr int HPT = (NHALO + NT - 1) / NT;
    static constexpr unsigned PLANE_BYTES = (unsigned)(NF * MAIN * sizeof(double));
    // kTmaSlots slots, one mbarrier each, 128 bytes of alignment slack
    static constexpr size_t smem_bytes = sizeof(double) * kTmaSlots * SLOT + kTmaSlots * 8 + 128;
    static_assert(TX * sizeof(double) % 16 == 0, "TMA box rows are whole 16-byte units");
    static_assert(TX <= 256 && ROWS <= 256, "TMA box dimensions");
};

template <int TX, int TY, bool GAUGED>
struct TmaStage {
    using T = double;
    using LY = TmaLayout<TX, TY, GAUGED>;
    static constexpr int NF = LY::NF;
    static constexpr int NSLOT = kTmaSlots;
    static constexpr bool MOM = false;   // momenta read from global memory at the site
    __device__ __forceinline__ void issue_mom(int, int) {}
    __device__ __forceinline__ void wait_mom(int) {}
    __device__ __forceinline__ double mom(int, int) const { return 0.0; }
    double *xs;
    unsigned bar0;           // shared address of the slot-0 mbarrier (slot s at bar0 + 8 s)
    unsigned phase = 0;      // bit s: parity of the next completion of slot s
    const TmaMaps *maps;
    int *flag;
    int N;
    long long N3;
    int k0, j0, edge;        // edge: 0 interior, 1 bottom (j0 = 0), 2 top (j0 + TY = N)
    int h_s[LY::HPT];        // this thread's halo-column doubles: shared offset in a slot,
    long long h_g[LY::HPT];  // offset in a plane of the buffer (field * N^3 + j * N + k), -1: none
    bool timed_out = false;

    __device__ __forceinline__ TmaStage(unsigned char *smem, const TmaMaps *m, int *fl) : maps(m), flag(fl) {
        // round up to 128 bytes by offsetting the shared array itself (an
        // integer round trip would hide the address space and turn every ring
        // read into a generic load)
        const unsigned off = (128u - (smem_u32(smem) & 127u)) & 127u;
        xs = reinterpret_cast<double *>(smem + off);
        bar0 = smem_u32(xs + kTmaSlots * LY::SLOT);
        if (threadIdx.x == 0) {
            for (int s = 0; s < kTmaSlots; s++) mbar_init(bar0 + 8 * s, 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncthreads();
    }

    __device__ __forceinline__ void begin(const StepConsts &c, int k0_, int j0_, int, int) {
        N = c.N;
        N3 = c.N3;
        k0 = k0_;
        j0 = j0_;
        edge = (j0 == 0) ? 1 : (j0 + TY == N ? 2 : 0);
        const int kl = wrapi(k0 - 1, N), kr = wrapi(k0 + TX, N);
#pragma unroll
        for (int q = 0; q < LY::HPT; q++) {
            const int e = threadIdx.x + q * LY::NT;
            int side = 0, row = 0, f = 0;
            h_g[q] = -1;
            h_s[q] = 0;
            if (e < 2 * TY * NF) {
                side = e / (TY * NF);
                const int rem = e - side * TY * NF;
                row = 1 + rem / NF;
                f = rem % NF;
            } else if (e < LY::NHALO) {   // corners: (row TY + 1, left) and (row 0, right), link angles only
                const int q3 = e - 2 * TY * NF;
                side = q3 / 3;
                row = side == 0 ? TY + 1 : 0;
                f = FTH + q3 % 3;
            } else {
                continue;
            }
            h_s[q] = f * LY::FS + (side == 0 ? LY::LEFT : LY::RIGHT) + row;
            h_g[q] = (long long)f * N3 + (long long)wrapi(j0 - 1 + row, N) * N + (side == 0 ? kl : kr);
        }
    }

    __device__ __forceinline__ void issue(const StepIO<F64> &io, int p, int slot) {
        const int pw = wrapi(p, N);
        double *sb = xs + slot * LY::SLOT;
        const unsigned bar = bar0 + 8 * slot;
        if (threadIdx.x < 32) {   // warp 0: one lane per field
            if (threadIdx.x == 0) mbar_expect_tx(bar, LY::PLANE_BYTES);
            __syncwarp();
            for (int f = threadIdx.x; f < NF; f += 32) {
                const unsigned dst = smem_u32(sb + f * LY::FS);
                if (edge == 0) {
                    tma_load_4d(dst, &maps->full, k0, j0 - 1, pw, f, bar);
                } else if (edge == 1) {   // rows j0 .. j0 + TY, then the wrapped row N - 1 on top
                    tma_load_4d(dst + TX * 8, &maps->part, k0, 0, pw, f, bar);
                    tma_load_4d(dst, &maps->row, k0, N - 1, pw, f, bar);
                } else {                  // rows j0 - 1 .. j0 + TY - 1, then the wrapped row 0 below
                    tma_load_4d(dst, &maps->part, k0, j0 - 1, pw, f, bar);
                    tma_load_4d(dst + (TY + 1) * TX * 8, &maps->row, k0, 0, pw, f, bar);
                }
            }
        }
        const double *gb = io.xin + (long long)pw * N * N;
#pragma unroll
        for (int q = 0; q < LY::HPT; q++)
            if (h_g[q] >= 0) cp_async8(sb + h_s[q], gb + h_g[q]);
    }
    __device__ __forceinline__ void commit() { cp_async_commit(); }
    // the block loads of slot s and this thread's halo copies (all but the
    // PENDING latest groups) have landed; a wait that gives up sets the
    // timeout bit and lets the launch finish
    template <int PENDING>
    __device__ __forceinline__ void wait(int s) {
        cp_async_wait<PENDING>();
        const unsigned par = (phase >> s) & 1u;
        unsigned n = 0;
        while (!mbar_try_wait(bar0 + 8 * s, par)) {
            if (++n >= kTmaWaitLimit) {
                if (!timed_out) atomicOr(flag, kFlagTimeout);
                timed_out = true;
                break;
            }
        }
        phase ^= 1u << s;
    }
    __device__ __forceinline__ double at(int slot, int f, int r, int col) const {
        const int off = (col == 0) ? LY::LEFT + r : (col == TX + 1 ? LY::RIGHT + r : r * TX + col - 1);
        return xs[slot * LY::SLOT + f * LY::FS + off];
    }
};

// The cp.async position ring with the momenta staged through TMA: one dense
// TX x TY box per field and plane (no halo, so no wrap and no split boxes),
// loaded one plane ahead into two slots with an mbarrier each, and read by
// each thread at its own site from shared memory instead of from global
// memory.  The tensor map covers the handle's momentum buffer that the launch
// reads (W, or S on the first launch).
template <int TX, int TY, bool GAUGED>
struct CpMomStage : CpStage<F64, TX, TY, GAUGED> {
    using Base = CpStage<F64, TX, TY, GAUGED>;
    static constexpr bool MOM = true;
    static constexpr int NF = Base::NF;
    static constexpr int MSLOT = NF * TX * TY;                    // doubles per momentum slot
    static constexpr unsigned MOM_BYTES = (unsigned)(MSLOT * sizeof(double));
    static constexpr size_t ring_bytes = Base::LY::smem_bytes;
    // position ring, 128 bytes of slack, 2 momentum slots, 2 mbarriers
    static constexpr size_t smem_bytes = ring_bytes + 128 + 2 * MOM_BYTES + 16;
    double *ms;
    unsigned mbar0;
    unsigned mphase = 0;
    const CUtensorMap *mmap;
    int *flag;
    int k0, j0;
    bool timed_out = false;

    __device__ __forceinline__ CpMomStage(unsigned char *smem, const CUtensorMap *m, int *fl)
        : Base(smem), mmap(m), flag(fl) {
        const unsigned base = smem_u32(smem);
        const unsigned off = ((base + (unsigned)ring_bytes + 127u) & ~127u) - base;
        ms = reinterpret_cast<double *>(smem + off);
        mbar0 = smem_u32(ms + 2 * MSLOT);
        if (threadIdx.x == 0) {
            mbar_init(mbar0, 1);
            mbar_init(mbar0 + 8, 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncthreads();
    }
    __device__ __forceinline__ void begin(const StepConsts &c, int k0_, int j0_, int nk, int nj) {
        Base::begin(c, k0_, j0_, nk, nj);
        k0 = k0_;
        j0 = j0_;
    }
    __device__ __forceinline__ void issue_mom(int p, int slot) {
        if (threadIdx.x < 32) {   // warp 0: one lane per field
            const unsigned bar = mbar0 + 8 * slot;
            if (threadIdx.x == 0) mbar_expect_tx(bar, MOM_BYTES);
            __syncwarp();
            for (int f = threadIdx.x; f < NF; f += 32)
                tma_load_4d(smem_u32(ms + slot * MSLOT + f * TX * TY), mmap, k0, j0, p, f, bar);
        }
    }
    __device__ __forceinline__ void wait_mom(int slot) {
        const unsigned par = (mphase >> slot) & 1u;
        unsigned n = 0;
        while (!mbar_try_wait(mbar0 + 8 * slot, par)) {
            if (++n >= kTmaWaitLimit) {
                if (!timed_out) atomicOr(flag, kFlagTimeout);
                timed_out = true;
                break;
            }
        }
        mphase ^= 1u << slot;
    }
    // this thread's momentum f (site (ty, tx) of the tile)
    __device__ __forceinline__ double mom(int slot, int f) const { return ms[slot * MSLOT + f * TX * TY + threadIdx.x]; }
};

template <int TX, int TY, bool GAUGED, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(TX * TY, (MinBlocks<F64, TX, TY, GAUGED>::value))
step_cpm_kernel(StepIO<F64> io, StepConsts c, TileGrid tg, const __grid_constant__ CUtensorMap mmap) {
    extern __shared__ __align__(16) unsigned char cpm_smem[];
    CpMomStage<TX, TY, GAUGED> stg(cpm_smem, &mmap, io.flag);
    bool stop = false;
    for_each_piece(tg, c.N, [&](const Piece &pc) {
        if (stop) return;
        step_item<F64, TX, TY, GAUGED, FIRST>(io, c, pc, SYNC, DAMP, stg);
        stop = __syncthreads_or(stg.timed_out);   // every thread leaves together
    });
}

template <int TX, int TY, bool GAUGED, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(TX * TY, (MinBlocks<F64, TX, TY, GAUGED>::value))
step_tma_kernel(StepIO<F64> io, StepConsts c, TileGrid tg, const __grid_constant__ TmaMaps maps) {
    extern __shared__ __align__(16) unsigned char tma_smem[];   // aligned to 128 bytes by TmaStage
    TmaStage<TX, TY, GAUGED> stg(tma_smem, &maps, io.flag);
    bool stop = false;
    for_each_piece(tg, c.N, [&](const Piece &pc) {
        if (stop) return;
        step_item<F64, TX, TY, GAUGED, FIRST>(io, c, pc, SYNC, DAMP, stg);
        stop = __syncthreads_or(stg.timed_out);   // every thread leaves together
    });
}

}  // namespace scp
