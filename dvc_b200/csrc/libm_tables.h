// Correction tables for exact_libm.h: file layout, host loader, device view.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
#include <vector>
#endif

#define XLM_MAGIC "DVCXLM02"

typedef struct {
  char magic[8];
  char libc[24];        // C library version the tables were swept from
  uint32_t log_cap, log_count;  // logf hash: log_cap (key, value) slots, power of two
  uint32_t exp_cap, exp_count;  // expf hash
  uint32_t tanh_ylo, tanh_y1;   // tanh argument range [ylo, y1) covered by the bitmap; y >= y1 gives 1
  uint32_t em1_words, em1_count;  // expm1f exception bitmap (u32 words over y - ylo)
  uint32_t esc_cap, esc_count;    // expm1f escapes (key y bits -> value) where the neighbour rule fails
  uint32_t reserved[4];
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
  const uint32_t *em1_bitmap;
  const uint32_t *esc_tab;
  uint32_t log_mask, exp_mask, esc_mask;  // cap - 1
  int log_shift, exp_shift, esc_shift;    // 32 - log2(cap)
  uint32_t tanh_ylo, tanh_y1;
  const XlmSmallTables *small;  // device copy
} XlmDev;

#ifdef __cplusplus
struct XlmHost {
  XlmHeader hdr;
  std::vector<uint32_t> log_tab, exp_tab, em1_bitmap, esc_tab;
  XlmSmallTables small;
};
extern "C" {
#endif
int dvc_libm_build(const char *path, int threads, char *err, int errlen);
#ifdef __cplusplus
}
int dvc_libm_load(const char *path, XlmHost *out, char *err, int errlen);
#endif
