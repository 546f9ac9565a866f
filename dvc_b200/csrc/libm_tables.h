// Correction tables for exact_libm.h: file layout, host loader, device view.
#pragma once
#include <stdint.h>
#include <vector_types.h>

#ifdef __cplusplus
#include <vector>
#endif

#define XLM_MAGIC "DVCXLM04"

typedef struct {
  char magic[8];
  char libc[24];        // C library version the tables were swept from
  uint32_t log_cap, log_count;  // logf hash: log_cap (key, value) slots, power of two
  uint32_t exp_cap, exp_count;  // expf hash
  uint32_t tanh_ylo, tanh_y1;   // tanh argument range [ylo, y1) of the phi table; y >= y1 gives tanhf 1
  uint32_t exp_tie;             // largest xl_tie_dist of an expf exception with a normal result
  uint32_t reserved[7];
} XlmHeader;

// small tables of the base functions (exact_libm.h); stored after the big ones
typedef struct {
  double exp2j[32];
  double invc[128];
  double logc[128];
  int efold[128];
} XlmSmallTables;

// Device-side view, passed by value to kernels.
typedef struct {
  const uint32_t *log_tab;
  const uint32_t *exp_tab;
  // -logf(tanhf(y)) for y bits in [tanh_ylo, tanh_y1), packed (exact_libm.h):
  const uint4 *phi_desc;  // per binade: first record, format, ceil(2^32 / G), 0
  const uint4 *phi_rec;   // 16-byte records
  int phi_nbin;           // binades (descriptors), at most XL_PHI_MAX_BINADES
  uint32_t log_mask, exp_mask;  // cap - 1
  int log_shift, exp_shift;     // 32 - log2(cap)
  uint32_t tanh_ylo, tanh_y1;
  uint32_t exp_tie;
  const XlmSmallTables *small;  // device copy
  // phi_rec as a texture object (cudaTextureObject_t; element reads, no
  // filtering): the BP kernels gather the records through the texture path,
  // which leaves the load/store path to their shared-memory traffic
  unsigned long long phi_tex;
} XlmDev;

#ifdef __cplusplus
struct XlmHost {
  XlmHeader hdr;
  std::vector<uint32_t> log_tab, exp_tab;
  XlmSmallTables small;
};
extern "C" {
#endif
int dvc_libm_build(const char *path, int threads, char *err, int errlen);
#ifdef __cplusplus
}
int dvc_libm_load(const char *path, XlmHost *out, char *err, int errlen);
// out[i] = -logf(tanhf(y)) with the C library, y the float with bits ylo + i, i < y1 - ylo
void dvc_phi_build(float *out, uint32_t ylo, uint32_t y1, int threads);

// packed form of that table (exact_libm.h): desc holds 4 words per binade,
// rec 4 words per record
struct PhiPacked {
  std::vector<uint32_t> desc, rec;
};
// Packs phi[0 .. y1 - ylo) (ylo must start a binade) and checks every entry
// of the packed table against phi; returns false with a message on failure.
bool dvc_phi_pack(const float *phi, uint32_t ylo, uint32_t y1, int threads, PhiPacked &out, char *err, int errlen);
#endif
