// Fused x pass with bulk-staged inputs (the warp-granular kernel's
// computation, for N = 256 and 512).
//
// Every warp runs line pairs in a loop.  The input half lines of the next
// round of inverse transforms (the SPW sequences of the round, two half lines
// each) are copied into a per-warp double buffer in shared memory by one lane
// with 1D bulk copies (cp.async.bulk, completion on an mbarrier), one round
// ahead; the copies of a pair's first round are issued during the previous
// pair's last inverse round, so they land while that pair's product, forward
// transforms and stores run.  No registers hold prefetched values, and no
// global load sits on a transform's critical path.  Rows are 16-byte aligned
// (the padded workspace pitch); with pruning only [0, kxa) rounded up to 16
// bytes and the Nyquist element are copied.  Waits are bounded: a wait that
// gives up sets the status flag, waits (bounded) for the warp's copies in
// flight and returns.
#pragma once

#include "kernels.cuh"
#include "tc.cuh"

namespace dnsbox {

template <typename T, int N> struct XlineBulk {
  using PL = typename XlineWarp<T, N>::Plan;
  using C = typename CT<T>::type;
  static constexpr bool on = XlineWarp<T, N>::on;
  static constexpr int P = N / PL::E;
  static constexpr int SPW = 32 / P;
  static constexpr int RND = 6 / SPW;                        // inverse rounds per pair
  static constexpr int LDC = N + N / PL::R[0];
  static constexpr int Q = 16 / (int)sizeof(C);              // complex per 16 bytes
  static constexpr int HP = (N / 2 + 1 + Q - 1) / Q * Q;     // staged complex per half line
  static constexpr int WPB = sizeof(T) == 8 && N >= 512 ? 1 : 2;
  static constexpr int WARP_ELEMS = 6 * LDC + 2 * SPW * 2 * HP;
  static constexpr size_t SMEM = (size_t)WPB * WARP_ELEMS * sizeof(C);
};

constexpr int kXlineWaitLimit = 1 << 22;

template <typename T, int N>
__global__ void __launch_bounds__(32 * XlineBulk<T, N>::WPB)
    k_xline_nl_wb(const __grid_constant__ XlineNLArgs<T> a) {
  using XB = XlineBulk<T, N>;
  using C = typename CT<T>::type;
  using PL = typename XB::PL;
  using EN = FftEndsP<PL>;
  using AD = AddrSkew<PL::R[0]>;
  constexpr int E = PL::E, P = XB::P, SPW = XB::SPW, RND = XB::RND, LDC = XB::LDC, HP = XB::HP, Q = XB::Q;
  constexpr int WPB = XB::WPB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mbar[WPB][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C *s = reinterpret_cast<C *>(smem_raw) + (size_t)warp * XB::WARP_ELEMS;
  C *stg = s + 6 * LDC;   // [buffer][SPW][2][HP]
  const long long npairs = a.nlines / 2, gw = (long long)blockIdx.x * WPB + warp, nw = (long long)gridDim.x * WPB;
  const long long pin = a.pin ? a.pin : a.nxh, pout = a.pout ? a.pout : a.nxh;
  if (lane == 0) {
    tc::mbar_init(&mbar[warp][0], 1);
    tc::mbar_init(&mbar[warp][1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (gw >= npairs) return;
  const long long myp = (npairs - gw + nw - 1) / nw;   // pairs of this warp
  const long long nrounds = myp * RND;
  // copy layout of a half line: [0, kl) and, when pruning, [N/2, N/2 + Q)
  const int kl = a.kxa ? ((a.kxa + Q - 1) / Q) * Q : HP;
  const uint32_t row_bytes = (uint32_t)(a.kxa ? (kl + Q) : HP) * (uint32_t)sizeof(C);
  // lane 0: issue the copies of round g into buffer g & 1
  auto issue = [&](long long g) {
    const long long pr = gw + (g / RND) * nw;
    const int r = (int)(g % RND);
    const long long la = 2 * pr, lb = la + 1;
    const C *f1s[6] = {a.U, a.U, a.W, a.OX, a.OX, a.OZ};
    const C *f2s[6] = {a.V, a.V, a.W, a.OY, a.OY, a.OZ};
    const long long l1s[6] = {la, lb, la, la, lb, la};
    const long long l2s[6] = {la, lb, lb, la, lb, lb};
    uint64_t *mb = &mbar[warp][g & 1];
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mb)),
                 "r"(row_bytes * 2u * SPW)
                 : "memory");
    C *buf = stg + (size_t)(g & 1) * SPW * 2 * HP;
    for (int hh = 0; hh < SPW; ++hh) {
      const int q = SPW * r + hh;
      for (int t = 0; t < 2; ++t) {
        const C *src = (t ? f2s[q] + l2s[q] * pin : f1s[q] + l1s[q] * pin);
        C *dst = buf + (size_t)(2 * hh + t) * HP;
        const uint32_t nlo = (uint32_t)kl * (uint32_t)sizeof(C);
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                tc::smem_u32(dst)),
            "l"(src), "r"(nlo), "r"(tc::smem_u32(mb))
            : "memory");
        if (a.kxa)
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  tc::smem_u32(dst + N / 2)),
              "l"(src + N / 2), "r"((uint32_t)(Q * sizeof(C))), "r"(tc::smem_u32(mb))
              : "memory");
      }
    }
  };
  if (lane == 0) issue(0);
  const int p = lane % P, h = lane / P;
  long long g = 0;   // round counter of this warp
  bool fail = false;
  for (long long k = 0; k < myp && !fail; ++k) {
    const long long pr = gw + k * nw;
    const long long la = 2 * pr, lb = la + 1;
#pragma unroll 1
    for (int r = 0; r < RND; ++r, ++g) {
      __syncwarp();   // round g - 1 has read buffer (g + 1) & 1
      if (lane == 0 && g + 1 < nrounds) {
        tc::fence_proxy_async();   // those reads before the bulk copies overwrite the buffer
        issue(g + 1);
      }
      const bool ok = tc::mbar_wait_bounded(&mbar[warp][g & 1], (uint32_t)(g >> 1) & 1u, kXlineWaitLimit);
      if (__any_sync(0xffffffffu, !ok)) {
        fail = true;
        break;
      }
      const C *buf = stg + (size_t)(g & 1) * SPW * 2 * HP + (size_t)(2 * h) * HP;
      const int q = SPW * r + h;
      C v[E];
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const int n = EN::in_row(p, i);
        const int kk = n <= N / 2 ? n : N - n;
        const bool kp = xkeep(a.kxa, kk, N);
        const C x1 = kp ? buf[kk] : mkc<C>(0, 0);
        const C x2 = kp ? buf[HP + kk] : mkc<C>(0, 0);
        v[i] = pack_pair<C, N>(n, x1, x2);
      }
      fft_regs_p<C, PL, true, true, AD>(v, s, LDC, q, p, true, a.tw);
#pragma unroll
      for (int i = 0; i < E; ++i) s[AD::at(EN::out_row(p, i), q, LDC)] = v[i];
    }
    if (fail) break;
    xline_w_tail<T, N>(s, a, la, lb, lane, pout);
  }
  if (fail && lane == 0) {
    // the copies in flight complete on the two barriers: wait for them (bounded)
    for (long long gg = g; gg < g + 2 && gg < nrounds; ++gg)
      tc::mbar_wait_bounded(&mbar[warp][gg & 1], (uint32_t)(gg >> 1) & 1u, kXlineWaitLimit);
    if (a.status) atomicExch(a.status, 1);
  }
}

}  // namespace dnsbox
