// Context creation: host-side table construction and upload.
//
// Replaces SetupConstants (reference src/ConstantsGPU.cu:132-640) and the CRT tables the
// reference takes from OpenFHE's raw parameters (RawCiphertext.cu:258-633):
//   - twiddles psi_rev[j] = psi^brev(j) with Shoup companions (ConstantsGPU.cu:246-318);
//   - ModUp tables PartQlHatInvModq / PartQlHatModp per (level, digit), digits being
//     OpenFHE's contiguous partition of alpha = ceil(n_q / dnum) primes (Context.cu:268-339);
//   - ModDown tables PHatInvModp / PHatModq / PInvModq (ConstantsGPU.cu:480-534);
//   - rescale constants q_l^-1 and QlQlInvModqlDivqlModq (RawCiphertext.cu:318-440), the
//     latter equal to -q_l^-1 mod q_j because q_j divides Q_{l-1}.
#include <cmath>
#include <algorithm>
#include <cstring>
#include <thread>

#include "context.hpp"
#include "conv_tc.hpp"

namespace fides {

typedef unsigned __int128 u128;

uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  for (; e; e >>= 1) {
    if (e & 1) r = h_mulmod(r, a, q);
    a = h_mulmod(a, a, q);
  }
  return r;
}
uint64_t h_invmod(uint64_t a, uint64_t q) { return h_powmod(a % q, q - 2, q); }

// Smallest primitive root g of q, then psi = g^((q-1)/2N) (the reference's standalone rule).
uint64_t h_root_2n(uint64_t q, int logN) {
  std::vector<uint64_t> fact;
  uint64_t phi = q - 1, n = phi;
  for (uint64_t i = 2; i * i <= n; ++i)
    if (n % i == 0) {
      fact.push_back(i);
      while (n % i == 0) n /= i;
    }
  if (n > 1) fact.push_back(n);
  uint64_t g = 2;
  for (;; ++g) {
    bool ok = true;
    for (uint64_t f : fact)
      if (h_powmod(g, phi / f, q) == 1) {
        ok = false;
        break;
      }
    if (ok) break;
  }
  return h_powmod(g, (q - 1) / (2ull << logN), q);
}

ShoupConst h_shoup(uint64_t w, uint64_t q) {
  ShoupConst c;
  c.w = w;
  c.ws = (uint64_t)(((u128)w << 64) / q);
  return c;
}

static uint32_t h_brev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

uint32_t h_auto_index(int logN, int rotation) {
  const int64_t N = 1ll << logN;
  if (rotation == 2 * N - 1) return (uint32_t)(2 * N - 1);
  int64_t h = N / 2, r = rotation % h;
  if (r < 0) r += h;
  return (uint32_t)h_powmod(5, (uint64_t)(2 * N - r), (uint64_t)(2 * N));
}

static bool h_is_prime(uint64_t n) {
  static const uint64_t b[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return false;
  for (uint64_t p : b) {
    if (n == p) return true;
    if (n % p == 0) return false;
  }
  uint64_t d = n - 1;
  int s = 0;
  while (!(d & 1)) d >>= 1, ++s;
  for (uint64_t a : b) {
    uint64_t x = h_powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s && comp; ++r) {
      x = h_mulmod(x, x, n);
      if (x == n - 1) comp = false;
    }
    if (comp) return false;
  }
  return true;
}

Scratch::Scratch(Context* c, size_t b, cudaStream_t st) : ctx(c), s(st), bytes(b) {
  if (b == 0) return;
  size_t now = ctx->scratch_in_use.fetch_add(b) + b;
  if (ctx->scratch_limit && now > ctx->scratch_limit) {
    ctx->scratch_in_use.fetch_sub(b);
    throw Error(-3, "scratch limit exceeded: need " + std::to_string(now) + " bytes, limit " +
                        std::to_string(ctx->scratch_limit));
  }
  size_t peak = ctx->scratch_peak.load();
  while (now > peak && !ctx->scratch_peak.compare_exchange_weak(peak, now)) {
  }
  cudaError_t e = cudaMallocFromPoolAsync(&p, b, ctx->pool, s);
  if (e != cudaSuccess) {
    ctx->scratch_in_use.fetch_sub(b);
    cudaGetLastError();
    throw Error(-3, std::string("device scratch allocation failed: ") + cudaGetErrorString(e));
  }
}

void reserve_scratch(Context* c, size_t bytes) {
  if (bytes == 0) return;
  FIDES_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = nullptr;
  FIDES_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, c->pool, s);
  if (e == cudaSuccess) e = cudaFreeAsync(p, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(-3, std::string("scratch reservation failed: ") + cudaGetErrorString(e));
  }
  FIDES_CUDA(e2);
}

Scratch::~Scratch() {
  if (p) {
    cudaFreeAsync(p, s);
    ctx->scratch_in_use.fetch_sub(bytes);
  }
}

static cudaEvent_t take_event(Context* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  FIDES_CUDA(cudaEventCreate(&e));
  return e;
}

LaunchScope::LaunchScope(Context* ctx, cudaStream_t st, int kind, double bytes) : c(ctx), s(st) {
  c->launches.fetch_add(1);
  if (!c->profiling) return;
  std::lock_guard<std::mutex> g(c->prof_mu);
  ProfileRec r{kind, take_event(c), take_event(c), bytes};
  FIDES_CUDA(cudaEventRecord(r.beg, s));
  c->prof.push_back(r);
  idx = (int)c->prof.size() - 1;
}

LaunchScope::~LaunchScope() {
  if (idx < 0) return;
  std::lock_guard<std::mutex> g(c->prof_mu);
  cudaEventRecord(c->prof[idx].end, s);
}

template <typename T>
static void append(std::vector<char>& blob, const std::vector<T>& v, size_t& off) {
  size_t a = 16;
  size_t o = (blob.size() + a - 1) / a * a;
  blob.resize(o + sizeof(T) * v.size());
  if (!v.empty()) std::memcpy(blob.data() + o, v.data(), sizeof(T) * v.size());
  off = o;
}

Context* create_context(int logN, int n_q, int K, int dnum, const uint64_t* primes, const uint64_t* psi, int device) {
  if (logN < 4 || logN > 17) throw Error(-1, "logN must be in [4, 17]");
  if (n_q < 1 || K < 0 || dnum < 1 || dnum > n_q) throw Error(-1, "need n_q >= 1, K >= 0, 1 <= dnum <= n_q");
  if (n_q + K > 256) throw Error(-1, "at most 256 primes");
  const int np = n_q + K;
  const uint64_t N = 1ull << logN;
  for (int i = 0; i < np; ++i) {
    uint64_t q = primes[i];
    if (q >= (1ull << 62) || q < 3 || (q - 1) % (2 * N) != 0 || !h_is_prime(q))
      throw Error(-1, "prime " + std::to_string(i) + " = " + std::to_string(q) +
                          " is not a prime < 2^62 with q = 1 mod 2N");
    for (int j = 0; j < i; ++j)
      if (primes[j] == q) throw Error(-1, "primes must be distinct");
  }
  auto* c = new Context();
  c->device = device;
  c->logN = logN;
  c->N = (int)N;
  c->n_q = n_q;
  c->K = K;
  c->dnum = dnum;
  c->alpha = (n_q + dnum - 1) / dnum;
  c->primes.assign(primes, primes + np);
  c->psi.resize(np);
  for (int i = 0; i < np; ++i) {
    uint64_t q = primes[i];
    uint64_t p = (psi && psi[i]) ? psi[i] : h_root_2n(q, logN);
    if (h_powmod(p, N, q) != q - 1) {
      delete c;
      throw Error(-1, "psi[" + std::to_string(i) + "] is not a primitive 2N-th root of unity");
    }
    c->psi[i] = p;
  }
  try {
    FIDES_CUDA(cudaSetDevice(device));
    // ---- per-prime constants and twiddles
    std::vector<DevPrime> hp(np);
    std::vector<ShoupConst> tf((size_t)np * N), ti((size_t)np * N), il(np);
    std::vector<double2> tff((size_t)np * N), tfi((size_t)np * N);
    std::vector<double> twf_w((size_t)np * N), twi_w((size_t)np * N);
    std::vector<F64Prime> f64(np);
    auto work = [&](int i) {
      uint64_t q = primes[i];
      DevPrime& d = hp[i];
      d.q = q;
      d.q2 = 2 * q;
      d.one_s = (uint64_t)(((u128)1 << 64) / q);
      d.r64 = (uint64_t)(((u128)1 << 64) % q);
      d.r64_s = h_shoup(d.r64, q).ws;
      d.ninv = h_invmod(N % q, q);
      d.ninv_s = h_shoup(d.ninv, q).ws;
      d.pad = 0;
      std::vector<uint64_t> pw(N), ipw(N);
      uint64_t ip = h_invmod(c->psi[i], q);
      pw[0] = ipw[0] = 1;
      for (uint64_t j = 1; j < N; ++j) {
        pw[j] = h_mulmod(pw[j - 1], c->psi[i], q);
        ipw[j] = h_mulmod(ipw[j - 1], ip, q);
      }
      for (uint64_t j = 0; j < N; ++j) {
        uint32_t r = h_brev((uint32_t)j, logN);
        tf[i * N + j] = h_shoup(pw[r], q);
        ti[i * N + j] = h_shoup(ipw[r], q);
      }
      il[i] = h_shoup(h_mulmod(ipw[h_brev(1, logN)], d.ninv, q), q);
      const double qd = (double)q;  // exact for q < 2^53; used only for q < 2^50
      for (size_t j = 0; j < (size_t)N; ++j) {
        tff[i * N + j] = make_double2((double)tf[i * N + j].w, (double)tf[i * N + j].w / qd);
        tfi[i * N + j] = make_double2((double)ti[i * N + j].w, (double)ti[i * N + j].w / qd);
        twf_w[i * N + j] = (double)tf[i * N + j].w / qd;  // correctly rounded w / q
        twi_w[i * N + j] = (double)ti[i * N + j].w / qd;
      }
      f64[i] = F64Prime{qd, 1.0 / qd, (double)d.ninv, (double)d.ninv / qd, (double)il[i].w, (double)il[i].w / qd};
    };
    {
      unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
      std::vector<std::thread> th;
      for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
          for (int i = (int)t; i < np; i += (int)nt) work(i);
        });
      for (auto& t : th) t.join();
    }
    // ---- P mod q_j, P^-1 mod q_j, rescale constants
    std::vector<ShoupConst> pinv(n_q), pmod(n_q);
    for (int j = 0; j < n_q; ++j) {
      uint64_t q = primes[j], P = 1;
      for (int k = 0; k < K; ++k) P = h_mulmod(P, primes[n_q + k] % q, q);
      pmod[j] = h_shoup(P, q);
      pinv[j] = h_shoup(h_invmod(P, q), q);
    }
    std::vector<RescaleConst> rs((size_t)(n_q + 1) * n_q);
    std::vector<ShoupConst> pqinv((size_t)(n_q + 1) * n_q, ShoupConst{0, 0});
    for (int l = 2; l <= n_q; ++l) {
      uint64_t qt = primes[l - 1];
      for (int j = 0; j < l - 1; ++j) {
        uint64_t q = primes[j];
        uint64_t qi = h_invmod(qt % q, q);
        uint64_t m = qi ? q - qi : 0;
        RescaleConst& r = rs[(size_t)l * n_q + j];
        ShoupConst a = h_shoup(qi, q), b = h_shoup(m, q);
        r.qinv = a.w;
        r.qinv_s = a.ws;
        r.m = b.w;
        r.m_s = b.ws;
        if (K > 0) pqinv[(size_t)l * n_q + j] = h_shoup(h_mulmod(pinv[j].w, qi, q), q);
      }
    }
    // ---- conversion tables
    struct HostConv {
      std::vector<int> src_pos, src_prime, dst_pos, dst_prime;
      std::vector<ShoupConst> pre;
      std::vector<uint64_t> mat;
      std::vector<uint8_t> tc_b;  // empty: no tensor-core form
      std::vector<TcDest> tc_dst;
      int kpad = 0, ndp = 0, lift = 0;
    };
    auto build_conv = [&](const std::vector<int>& sp, const std::vector<int>& spr, const std::vector<int>& dp,
                          const std::vector<int>& dpr, int lift) {
      HostConv h;
      h.src_pos = sp;
      h.src_prime = spr;
      h.dst_pos = dp;
      h.dst_prime = dpr;
      h.lift = lift;
      int ns = (int)spr.size(), nd = (int)dpr.size();
      h.pre.resize(ns);
      h.mat.resize((size_t)(ns + lift) * nd);
      for (int j = 0; j < nd && lift; ++j) {  // row ns: [-Q_src]_{p_j} (reference ReducedNoiseConstants.cu)
        uint64_t pj = primes[dpr[j]], v = 1 % pj;
        for (int k = 0; k < ns; ++k) v = h_mulmod(v, primes[spr[k]] % pj, pj);
        h.mat[(size_t)ns * nd + j] = v ? pj - v : 0;
      }
      for (int i = 0; i < ns; ++i) {
        uint64_t qi = primes[spr[i]], hq = 1;
        for (int k = 0; k < ns; ++k)
          if (k != i) hq = h_mulmod(hq, primes[spr[k]] % qi, qi);
        h.pre[i] = h_shoup(h_invmod(hq, qi), qi);
        for (int j = 0; j < nd; ++j) {
          uint64_t pj = primes[dpr[j]], v = 1 % pj;
          for (int k = 0; k < ns; ++k)
            if (k != i) v = h_mulmod(v, primes[spr[k]] % pj, pj);
          h.mat[(size_t)i * nd + j] = v;
        }
      }
      if (conv_tc_fits(logN, ns + lift, nd, primes, dpr))
        build_tc_image(h.mat.data(), ns + lift, nd, dpr, primes, h.tc_b, h.tc_dst, h.kpad, h.ndp);
      return h;
    };
    // [lift][l]: the plain tables and the reduced-noise ones
    std::vector<std::vector<HostConv>> hmu[2] = {std::vector<std::vector<HostConv>>(n_q + 1),
                                                 std::vector<std::vector<HostConv>>(n_q + 1)};
    std::vector<HostConv> hmd[2] = {std::vector<HostConv>(n_q + 1), std::vector<HostConv>(n_q + 1)};
    for (int lift = 0; lift < 2; ++lift)
      for (int l = 1; l <= n_q; ++l) {
        int b = c->beta(l);
        for (int d = 0; d < b; ++d) {
          int s0 = d * c->alpha, s1 = std::min((d + 1) * c->alpha, l);
          std::vector<int> sp, spr, dp, dpr;
          for (int i = s0; i < s1; ++i) sp.push_back(i), spr.push_back(i);
          for (int i = 0; i < l; ++i)
            if (i < s0 || i >= s1) dp.push_back(i), dpr.push_back(i);
          for (int k = 0; k < K; ++k) dp.push_back(l + k), dpr.push_back(n_q + k);
          hmu[lift][l].push_back(build_conv(sp, spr, dp, dpr, lift));
        }
        if (K > 0) {
          std::vector<int> sp, spr, dp, dpr;
          for (int k = 0; k < K; ++k) sp.push_back(k), spr.push_back(n_q + k);
          for (int j = 0; j < l; ++j) dp.push_back(j), dpr.push_back(j);
          hmd[lift][l] = build_conv(sp, spr, dp, dpr, lift);
        }
      }
    // ---- pack everything into one device blob
    std::vector<char> blob;
    size_t o_prime, o_tf, o_ti, o_il, o_pinv, o_pmod, o_rs, o_pq, o_tff, o_tfi, o_f64, o_tww, o_twwi;
    append(blob, hp, o_prime);
    append(blob, tf, o_tf);
    append(blob, ti, o_ti);
    append(blob, il, o_il);
    append(blob, pinv, o_pinv);
    append(blob, pmod, o_pmod);
    append(blob, rs, o_rs);
    append(blob, pqinv, o_pq);
    append(blob, tff, o_tff);
    append(blob, tfi, o_tfi);
    append(blob, twf_w, o_tww);
    append(blob, twi_w, o_twwi);
    append(blob, f64, o_f64);
    struct Off {
      size_t sp, spr, pre, dp, dpr, mat, tcb, tcd;
      int ns, nd, kpad, ndp, lift;
    };
    auto put = [&](const HostConv& h) {
      Off o;
      append(blob, h.src_pos, o.sp);
      append(blob, h.src_prime, o.spr);
      append(blob, h.pre, o.pre);
      append(blob, h.dst_pos, o.dp);
      append(blob, h.dst_prime, o.dpr);
      append(blob, h.mat, o.mat);
      append(blob, h.tc_b, o.tcb);
      append(blob, h.tc_dst, o.tcd);
      o.ns = (int)h.src_prime.size();
      o.nd = (int)h.dst_prime.size();
      o.kpad = h.tc_b.empty() ? 0 : h.kpad;
      o.ndp = h.ndp;
      o.lift = h.lift;
      return o;
    };
    std::vector<std::vector<Off>> omu[2] = {std::vector<std::vector<Off>>(n_q + 1),
                                            std::vector<std::vector<Off>>(n_q + 1)};
    std::vector<Off> omd[2] = {std::vector<Off>(n_q + 1), std::vector<Off>(n_q + 1)};
    for (int lift = 0; lift < 2; ++lift)
      for (int l = 1; l <= n_q; ++l) {
        for (auto& h : hmu[lift][l]) omu[lift][l].push_back(put(h));
        if (K > 0) omd[lift][l] = put(hmd[lift][l]);
      }
    FIDES_CUDA(cudaMalloc(&c->d_tables, blob.size()));
    FIDES_CUDA(cudaMemcpy(c->d_tables, blob.data(), blob.size(), cudaMemcpyHostToDevice));
    char* base = static_cast<char*>(c->d_tables);
    c->d_prime = reinterpret_cast<DevPrime*>(base + o_prime);
    c->d_tw_fwd = reinterpret_cast<ShoupConst*>(base + o_tf);
    c->d_tw_inv = reinterpret_cast<ShoupConst*>(base + o_ti);
    c->d_inv_last = reinterpret_cast<ShoupConst*>(base + o_il);
    c->d_pinv = reinterpret_cast<ShoupConst*>(base + o_pinv);
    c->d_pmod = reinterpret_cast<ShoupConst*>(base + o_pmod);
    c->d_rescale = reinterpret_cast<RescaleConst*>(base + o_rs);
    c->d_pqinv = reinterpret_cast<ShoupConst*>(base + o_pq);
    c->d_twf_fwd = reinterpret_cast<double2*>(base + o_tff);
    c->d_twf_inv = reinterpret_cast<double2*>(base + o_tfi);
    c->d_tww_fwd = reinterpret_cast<double*>(base + o_tww);
    c->d_tww_inv = reinterpret_cast<double*>(base + o_twwi);
    c->d_f64 = reinterpret_cast<F64Prime*>(base + o_f64);
    auto mk = [&](const Off& o) {
      ConvTable t;
      t.n_src = o.ns;
      t.n_dst = o.nd;
      t.src_pos = reinterpret_cast<const int*>(base + o.sp);
      t.src_prime = reinterpret_cast<const int*>(base + o.spr);
      t.pre = reinterpret_cast<const ShoupConst*>(base + o.pre);
      t.dst_pos = reinterpret_cast<const int*>(base + o.dp);
      t.dst_prime = reinterpret_cast<const int*>(base + o.dpr);
      t.mat = reinterpret_cast<const uint64_t*>(base + o.mat);
      t.lift = o.lift;
      if (o.kpad) {
        t.tc_b = reinterpret_cast<const uint8_t*>(base + o.tcb);
        t.tc_dst = reinterpret_cast<const TcDest*>(base + o.tcd);
        t.tc_kpad = o.kpad;
        t.tc_nd_pad = o.ndp;
      }
      return t;
    };
    c->modup_tab.resize(n_q + 1);
    c->moddown_tab.resize(n_q + 1);
    c->modup_tab_rn.resize(n_q + 1);
    c->moddown_tab_rn.resize(n_q + 1);
    for (int l = 1; l <= n_q; ++l) {
      for (auto& o : omu[0][l]) c->modup_tab[l].push_back(mk(o));
      for (auto& o : omu[1][l]) c->modup_tab_rn[l].push_back(mk(o));
      if (K > 0) {
        c->moddown_tab[l] = mk(omd[0][l]);
        c->moddown_tab_rn[l] = mk(omd[1][l]);
      }
    }
    // ---- scratch pool: keep freed blocks cached for reuse
    FIDES_CUDA(cudaDeviceGetDefaultMemPool(&c->pool, device));
    uint64_t thr = UINT64_MAX;
    FIDES_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr));
    FIDES_CUDA(cudaMalloc(&c->d_status, sizeof(uint32_t)));
    FIDES_CUDA(cudaMemset(c->d_status, 0, sizeof(uint32_t)));
    // ---- special-FFT twiddles for slot encode / decode (stage len = 2h, position j < h)
    {
      const size_t nh = (size_t)c->N / 2;
      std::vector<double> tw(2 * nh, 0.0);
      for (size_t h = 1; h < nh; h <<= 1) {
        const uint64_t m4 = 8 * h;  // 4 len
        uint64_t e = 1;             // 5^j mod 4 len
        for (size_t j = 0; j < h; ++j) {
          const double ang = -2.0 * M_PI * (double)e / (double)m4;
          tw[2 * (h + j)] = std::cos(ang);
          tw[2 * (h + j) + 1] = std::sin(ang);
          e = (e * 5) % m4;
        }
      }
      FIDES_CUDA(cudaMalloc(&c->d_sfft, tw.size() * sizeof(double)));
      FIDES_CUDA(cudaMemcpy(c->d_sfft, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  } catch (...) {
    destroy_context(c);
    throw;
  }
  return c;
}

void destroy_context(Context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (auto& r : c->prof) {
    cudaEventDestroy(r.beg);
    cudaEventDestroy(r.end);
  }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->d_tables) cudaFree(c->d_tables);
  if (c->d_status) cudaFree(c->d_status);
  if (c->d_sfft) cudaFree(c->d_sfft);
  if (c->pinned) cudaFreeHost(c->pinned);
  delete c;
}

}  // namespace fides
