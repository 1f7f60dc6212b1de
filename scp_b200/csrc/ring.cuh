// ring.cuh -- plane-ring tile walker of the extension steppers (Higgs and
// second gauge, three fabrics, the real mode's optional terms).
//
// Work is split as the fused step's: (TX x TY) columns of sites in (k, j)
// times segments of planes along i (TileGrid items).  A CTA streams its
// column plane by plane through a four-slot shared-memory ring that holds
// planes i-1, i, i+1 of every staged field, each with a one-site halo in j
// and k (corners included), while plane i+2 is in flight through cp.async.
// Each thread owns one site of the column; the halo sites of a plane are
// shared out one per thread among the first threads of the CTA.  With all
// three planes resident a model reads any of the 27 sites around its own
// from shared memory, so nothing is carried in registers from plane to
// plane unless the model chooses to.
//
// A model supplies
//   NR                 staged fields (each an N^3 array, site (i*N + j)*N + k)
//   Args               kernel arguments, with `RingSrc<NR> src` and `int N`
//   Carry              per-thread state kept along the i walk
//   site(args, view, i, j, k, idx, carry, first)   the work at one site
//   prefetch(args, idx)  L2 prefetch of what site() will read from global
//                        memory at idx on the next plane (its momenta), so the
//                        loads at the end of the next site update hit L2
// and runs as ring_kernel<Model, TX, TY>.
#pragma once
#include "common.cuh"

namespace scp {

template <int NR>
struct RingSrc {
    const double *f[NR];
    int prefetch = 1;   // 0: no L2 prefetch of the next plane's momenta
};

template <int NR, int TX, int TY>
struct RingShape {
    static constexpr int PX = TX + 2, PY = TY + 2;
    static constexpr int FIELD = PY * PX;          // elements of one field in one slot
    static constexpr int SLOT = NR * FIELD;
    static constexpr int NSLOT = 4;
    static constexpr int NT = TX * TY;
    static constexpr int MAXHALO = 2 * TX + 2 * TY + 4;
    static_assert(MAXHALO <= NT, "one halo site per thread at most");
    static constexpr size_t smem_bytes = sizeof(double) * NSLOT * SLOT;
};

// Read access to the three resident planes around one thread's site.
template <int NR, int TX, int TY>
struct RingView {
    using S = RingShape<NR, TX, TY>;
    const double *m, *c, *p;   // planes i-1, i, i+1 at this thread's site, field 0
    // field f at (i + di, j + dj, k + dk), di, dj, dk in {-1, 0, 1}
    __device__ __forceinline__ double at(int f, int di, int dj, int dk) const {
        const double *b = di < 0 ? m : (di > 0 ? p : c);
        return b[f * S::FIELD + dj * S::PX + dk];
    }
    __device__ __forceinline__ double operator()(int f) const { return c[f * S::FIELD]; }
};

// One work item of model M; extra arguments (a reduction's per-thread sums)
// are passed on to M::site.
template <class M, int TX, int TY, class... Extra>
__device__ __forceinline__ void ring_item(const typename M::Args &a, const Piece &pc, double *ring,
                                          Extra &...extra) {
    using S = RingShape<M::NR, TX, TY>;
    constexpr int NR = M::NR;
    const int N = a.N;
    const long long NN = (long long)N * N;
    const int k0 = pc.kt * TX, j0 = pc.jt * TY;
    const int i0 = pc.i0, i1 = pc.i1;
    const int nk = min(TX, N - k0), nj = min(TY, N - j0);
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const bool own = (tx < nk) && (ty < nj);
    const int k = k0 + tx, j = j0 + ty;
    const int own_s = (ty + 1) * S::PX + tx + 1;   // this site in a slot
    const int own_g = j * N + k;                    // and in a plane
    // the halo site this thread copies: rows j0-1 and j0+nj, columns k0-1 and
    // k0+nk, four corners; -1 when it has none
    int halo_s = -1, halo_g = 0;
    {
        const int h = tid;
        int r = -1, col = 0;
        if (h < nk) { r = 0; col = h + 1; }
        else if (h < 2 * nk) { r = nj + 1; col = h - nk + 1; }
        else if (h < 2 * nk + nj) { r = h - 2 * nk + 1; col = 0; }
        else if (h < 2 * nk + 2 * nj) { r = h - 2 * nk - nj + 1; col = nk + 1; }
        else if (h < 2 * nk + 2 * nj + 4) {
            const int q = h - 2 * nk - 2 * nj;
            r = (q & 1) ? nj + 1 : 0;
            col = (q & 2) ? nk + 1 : 0;
        }
        if (r >= 0) {
            halo_s = r * S::PX + col;
            halo_g = wrapi(j0 - 1 + r, N) * N + wrapi(k0 - 1 + col, N);
        }
    }
    auto stage = [&](int plane, int slot) {
        const long long pb = (long long)wrapi(plane, N) * NN;
        double *sb = ring + slot * S::SLOT;
#pragma unroll
        for (int f = 0; f < NR; f++) {
            if (own) cp_async8(sb + f * S::FIELD + own_s, a.src.f[f] + pb + own_g);
            if (halo_s >= 0) cp_async8(sb + f * S::FIELD + halo_s, a.src.f[f] + pb + halo_g);
        }
    };

    __syncthreads();   // the previous item's last plane has been read
    stage(i0 - 1, 0);
    stage(i0, 1);
    stage(i0 + 1, 2);
    cp_async_commit();
    typename M::Carry carry;
    for (int i = i0; i < i1; i++) {
        const int q = i - i0;
        cp_async_wait<0>();
        __syncthreads();   // planes i-1..i+1 are visible; slot (q+3)&3 (plane i-2) is free
        if (i + 2 <= i1) stage(i + 2, (q + 3) & 3);
        cp_async_commit();
        if (own) {
            RingView<NR, TX, TY> v;
            v.m = ring + (q & 3) * S::SLOT + own_s;
            v.c = ring + ((q + 1) & 3) * S::SLOT + own_s;
            v.p = ring + ((q + 2) & 3) * S::SLOT + own_s;
            if (a.src.prefetch && i + 1 < i1) M::prefetch(a, (long long)(i + 1) * NN + own_g);
            M::site(a, v, i, j, k, (long long)i * NN + own_g, carry, q == 0, extra...);
        }
    }
}

template <class M, int TX, int TY>
__global__ void __launch_bounds__(TX *TY, M::MIN_CTAS) ring_kernel(typename M::Args a, TileGrid tg) {
    extern __shared__ __align__(16) double ring[];
    for_each_piece(tg, a.N, [&](const Piece &pc) { ring_item<M, TX, TY>(a, pc, ring); });
}

__device__ __forceinline__ void prefetch_l2(const void *p) { prefetch_line_l2(p); }

// sponge factor 1 - rate * s^2 of the absorbing boundary at site (i, j, k),
// 1 inside radius L - width (apply_damping, sfa/sim/scp_sim.c:1440-1473)
__device__ __forceinline__ double sponge_at(int i, int j, int k, double L, double dx, double width, double rate) {
    const double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
    const double r = sqrt(x * x + y * y + z * z);
    const double inner = L - width;
    if (!(r > inner)) return 1.0;
    const double s = fmin((r - inner) / width, 1.0);
    return 1.0 - rate * s * s;
}

// Leapfrog update of one momentum / position pair in the fused scheme of the
// main step (state between launches: x_{n+1} and w_n = v_n + hdt a_n):
//   v_{n+1} = (w_n + hdt a) * damp,  w_{n+1} = v_{n+1} + hdt a,  x_{n+2} = x_{n+1} + dt w_{n+1}.
// A FIRST launch reads v_0 in place of w and takes no closing kick.
struct Leap {
    double hdt, dt;
    bool first;
    __device__ __forceinline__ void operator()(double w, double acc, double damp, double *v, double *wn) const {
        double vv = first ? w : w + hdt * acc;
        if (!first && damp != 1.0) vv *= damp;
        *v = vv;
        *wn = vv + hdt * acc;
    }
};

}  // namespace scp
