// Decoder context set-up.  See context.h.
#include "context.h"
#include "exact_libm.h"

#include <stdio.h>
#include <stdlib.h>
#include <sys/stat.h>

#include "kernels.h"

namespace dvc {

bool DevBuf::ensure(size_t b) {
  if (b <= bytes && p) return true;
  release();
  if (cudaMalloc(&p, b ? b : 16) != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return false;
  }
  bytes = b;
  return true;
}

bool DevBuf::ensure(size_t b, cudaStream_t stream) {
  if (!stream) return ensure(b);
  if (b <= bytes && p) return true;
  if (p) cudaFreeAsync(p, stream);
  p = nullptr;
  bytes = 0;
  if (cudaMallocAsync(&p, b ? b : 16, stream) != cudaSuccess) {
    p = nullptr;
    return false;
  }
  bytes = b;
  return true;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

bool Context::cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

static bool file_exists(const std::string &p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

bool Context::init(const char *data, const char *tables, int dev) {
  device = dev;
  data_dir = data ? data : "";
  table_dir = tables ? tables : data_dir;
  mkdir(table_dir.c_str(), 0755);
  if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return false;
  if (!cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
  // process-wide, set by every context creation: CIF 1024 unless the variable
  // asks for 512, QCIF 1024 unless it asks for 256 or 512
  const char *nt = getenv("DVC_LDPCA_THREADS");
  const char *ntq = getenv("DVC_LDPCA_THREADS_QCIF");
  set_ldpca_threads(nt ? atoi(nt) : 1024, ntq ? atoi(ntq) : 1024);
  // the same for the motion searches: threads per updateSI and forward-search block
  const char *si = getenv("DVC_SI_THREADS");
  const char *fme = getenv("DVC_FME_THREADS");
  set_me_shapes(si ? atoi(si) : 64, fme ? atoi(fme) : 256);

  // library-exact math tables: load, or sweep the C library once and cache
  const std::string xpath = table_dir + "/xlm_tables.bin";
  char ebuf[256] = {0};
  if (dvc_libm_load(xpath.c_str(), &xlm_host, ebuf, sizeof ebuf) != 0) {
    fprintf(stderr, "dvc_b200: building C-library correction tables (%s)\n", ebuf);
    if (dvc_libm_build(xpath.c_str(), 0, ebuf, sizeof ebuf) != 0) return fail(std::string("libm table build: ") + ebuf);
    if (dvc_libm_load(xpath.c_str(), &xlm_host, ebuf, sizeof ebuf) != 0) return fail(std::string("libm table load: ") + ebuf);
  }
  auto up = [&](const std::vector<uint32_t> &v, const uint32_t **dst) {
    void *p = nullptr;
    if (cudaMalloc(&p, v.size() * 4) != cudaSuccess) return false;
    xlm_allocs.push_back(p);
    if (cudaMemcpy(p, v.data(), v.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) return false;
    *dst = (const uint32_t *)p;
    return true;
  };
  if (!up(xlm_host.log_tab, &xlm.log_tab) || !up(xlm_host.exp_tab, &xlm.exp_tab))
    return fail("uploading libm tables failed");
  {
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(XlmSmallTables)) != cudaSuccess) return fail("uploading libm tables failed");
    xlm_allocs.push_back(p);
    if (cudaMemcpy(p, &xlm_host.small, sizeof(XlmSmallTables), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail("uploading libm tables failed");
    xlm.small = (const XlmSmallTables *)p;
  }
  auto lg2 = [](uint32_t v) {
    int s = 0;
    while ((1u << s) < v) s++;
    return s;
  };
  xlm.log_mask = xlm_host.hdr.log_cap - 1;
  xlm.exp_mask = xlm_host.hdr.exp_cap - 1;
  xlm.log_shift = 32 - lg2(xlm_host.hdr.log_cap);
  xlm.exp_shift = 32 - lg2(xlm_host.hdr.exp_cap);
  xlm.exp_tie = xlm_host.hdr.exp_tie;
  xlm.tanh_ylo = xlm_host.hdr.tanh_ylo;
  xlm.tanh_y1 = xlm_host.hdr.tanh_y1;
  {
    // phi = -logf(tanhf(y)) for every float y in [tanh_ylo, tanh_y1), from the
    // C library, swept and stored packed (every packed entry checked against the sweep)
    const size_t count = (size_t)xlm.tanh_y1 - xlm.tanh_ylo;
    PhiPacked pk;
    {
      std::vector<float> phi(count);
      dvc_phi_build(phi.data(), xlm.tanh_ylo, xlm.tanh_y1, 0);
      char perr[256];
      if (!dvc_phi_pack(phi.data(), xlm.tanh_ylo, xlm.tanh_y1, 0, pk, perr, sizeof perr)) return fail(perr);
    }
    if (pk.desc.size() / 4 > XL_PHI_MAX_BINADES) return fail("phi table has too many binades");
    auto put = [&](const void *src, size_t bytes, const void **dst) {
      void *p = nullptr;
      if (cudaMalloc(&p, bytes) != cudaSuccess) return false;
      xlm_allocs.push_back(p);
      if (cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return false;
      *dst = p;
      return true;
    };
    if (!put(pk.desc.data(), pk.desc.size() * 4, (const void **)&xlm.phi_desc) ||
        !put(pk.rec.data(), pk.rec.size() * 4, (const void **)&xlm.phi_rec))
      return fail("uploading the phi table failed");
    xlm.phi_nbin = (int)(pk.desc.size() / 4);
    {
      int max_linear = 0;
      cudaDeviceGetAttribute(&max_linear, cudaDevAttrMaxTexture1DLinearWidth, device);
      if ((size_t)max_linear < pk.rec.size() / 4) return fail("phi table exceeds the linear texture limit");
      cudaResourceDesc rd = {};
      rd.resType = cudaResourceTypeLinear;
      rd.res.linear.devPtr = const_cast<uint4 *>(xlm.phi_rec);
      rd.res.linear.desc = cudaCreateChannelDesc<uint4>();
      rd.res.linear.sizeInBytes = pk.rec.size() * 4;
      cudaTextureDesc td = {};
      td.readMode = cudaReadModeElementType;
      cudaTextureObject_t tex = 0;
      if (cudaCreateTextureObject(&tex, &rd, &td, nullptr) != cudaSuccess) return fail("phi texture object");
      xlm.phi_tex = tex;
    }
    phi_bytes = (pk.desc.size() + pk.rec.size()) * 4;
    // optional L2 persisting window over the records of the binades most BP
    // reads land in (y in [2^-6, 8), exponents 121..129: about 99% of the reads,
    // 60 MB), so that other kernels' streaming data does not evict them;
    // DVC_PHI_L2_MB = the set-aside in MB (0 or unset: off)
    set_phi_window(nullptr, 0, 0.0f);
    if (const char *mb = getenv("DVC_PHI_L2_MB")) {
      const size_t want = (size_t)atoi(mb) << 20;
      const int b_lo = 121 - (int)(xlm.tanh_ylo >> 23), b_hi = 129 - (int)(xlm.tanh_ylo >> 23);
      if (want > 0 && b_lo >= 0 && b_hi < xlm.phi_nbin) {
        const size_t r0 = pk.desc[4 * b_lo], r1 = b_hi + 1 < xlm.phi_nbin ? pk.desc[4 * (b_hi + 1)] : pk.rec.size() / 4;
        int max_persist = 0, max_window = 0;
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device);
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, device);
        size_t bytes = (r1 - r0) * 16, aside = want;
        if (bytes > (size_t)max_window) bytes = (size_t)max_window;
        if (aside > (size_t)max_persist) aside = (size_t)max_persist;
        if (bytes > 0 && aside > 0 && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, aside) == cudaSuccess)
          set_phi_window(xlm.phi_rec + r0, bytes, aside >= bytes ? 1.0f : (float)aside / (float)bytes);
        cudaGetLastError();
      }
    }
  }

  if (!near_ties.ensure(8) || !cuda_ok(cudaMemset(near_ties.p, 0, 8), "near-tie counter"))
    return fail("device allocation failed");

  // LDPCA ladders (QCIF n=1584 and CIF n=6336)
  const std::string lpath = data_dir + "/ldpca_ladders.bin";
  if (!file_exists(lpath)) return fail("missing ladder file " + lpath);
  if (!load_ladders(lpath, ladders_host, err)) return false;
  ladders_gpu.resize(ladders_host.size());
  for (size_t i = 0; i < ladders_host.size(); i++) {
    LadderHost &L = ladders_host[i];
    const std::string cache = table_dir + "/invh_" + std::to_string(L.n) + ".bin";
    if (!ladder_inverse(L, cache, err)) return false;
    if (!ladders_gpu[i].upload(L, err)) return false;
  }
  return true;
}

void Context::release() {
  for (auto &g : ladders_gpu) g.release();
  ladders_gpu.clear();
  if (xlm.phi_tex) cudaDestroyTextureObject((cudaTextureObject_t)xlm.phi_tex);
  xlm.phi_tex = 0;
  for (void *p : xlm_allocs) cudaFree(p);
  xlm_allocs.clear();
  ld_lr.release();
  ld_acc.release();
  ld_dec.release();
  ld_res.release();
  ld_ent.release();
  ld_jobs.release();
  near_ties.release();
  for (DevBuf *b : {&bt_lr, &bt_acc, &bt_dec, &bt_res, &bt_ent, &bt_cw, &bt_state}) b->release();
  if (stream) cudaStreamDestroy(stream);
  stream = nullptr;
}

const LadderDev *Context::ladder(int n) const {
  for (size_t i = 0; i < ladders_host.size(); i++)
    if (ladders_host[i].n == n) return &ladders_gpu[i].dev;
  return nullptr;
}

const LadderHost *Context::ladder_host(int n) const {
  for (auto &L : ladders_host)
    if (L.n == n) return &L;
  return nullptr;
}

}  // namespace dvc
