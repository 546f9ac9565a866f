// Test infrastructure: C entry points around the reference's own JBIG code
// (JBIG-KIT as vendored by the reference, with its simple_JBIG_enc /
// simple_JBIG_dec wrappers), used by the tests to pin the JBIG mode-map
// decoder of this library.  Built twice by oracle/Makefile:
//   -DJBIGREF_ENC with the encoder's objects  -> _ref/libjbigenc.so
//   -DJBIGREF_DEC with the decoder's objects  -> _ref/libjbigdec.so
// Maps are w x h bytes (0/1), row-major; the coded form is what the reference
// writes into the WZ bitstream (DvcEnc/src/wzbitstream.cpp:28-44) and reads
// back (DvcDec/src/wzbitstream.cpp:38-66).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "jbig.h"

#ifdef JBIGREF_ENC
unsigned char *BitToBitmap(unsigned char *Bits, int width, int height, int *numBytes);
int simple_JBIG_enc(FILE *fp, unsigned char *jbigdata, int width, int height, unsigned char jbgh[20], int stripe,
                    int write);

// coded bytes of the map into out[cap]; returns their count, -1 if cap is too small
extern "C" int jbigref_encode(const unsigned char *bits, int w, int h, unsigned char *out, int cap) {
  int nbytes = 0;
  unsigned char *bm = BitToBitmap(const_cast<unsigned char *>(bits), w, h, &nbytes);
  FILE *f = tmpfile();
  unsigned char jbgh[20];
  simple_JBIG_enc(f, bm, w, h, jbgh, h, 1);
  free(bm);
  const long n = ftell(f);
  rewind(f);
  int r = -1;
  if (n <= cap && fread(out, 1, (size_t)n, f) == (size_t)n) r = (int)n;
  fclose(f);
  return r;
}
#endif

#ifdef JBIGREF_DEC
unsigned char *ByteToBitmap(unsigned char *Bytes, int width, int height);
int simple_JBIG_dec(unsigned char *bdm_data, long int bdm_rsize, unsigned char jbgh[20], int total_len,
                    unsigned char *bdm_buffer);

// decode as the reference decoder does; returns the bytes consumed
extern "C" int jbigref_decode(const unsigned char *data, int len, int w, int h, unsigned char *bits) {
  const int buffer_size = (((((w + 4) >> 3) << 3) * h) >> 3) * 2;
  struct jbg_enc_state se;
  jbg_enc_init(&se, w, h, 1, NULL, NULL, NULL);
  jbg_enc_options(&se, JBG_ILEAVE | JBG_SMID, JBG_TPDON | JBG_DPON, h, 8, 0);
  unsigned char jbgh[20];
  jbg_set_header(&se, jbgh);
  unsigned char *in = (unsigned char *)calloc((size_t)buffer_size + 64, 1);
  unsigned char *dec = (unsigned char *)calloc((size_t)buffer_size + 64, 1);
  memcpy(in, data, (size_t)(len < buffer_size ? len : buffer_size));
  const int used = simple_JBIG_dec(in, buffer_size, jbgh, buffer_size, dec);
  unsigned char *b = ByteToBitmap(dec, w, h);
  memcpy(bits, b, (size_t)w * h);
  free(b);
  free(in);
  free(dec);
  return used;
}
#endif
