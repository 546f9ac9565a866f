// dvcdec: a DvcDec-compatible host executable over libdvc_b200.
//
//   dvcdec -d <decoder.cfg> [-Name=Value ...] [-GPUid=n] [-startFrame=a -endFrame=b]
//
// Same configuration keys and flags as the reference decoder
// (DvcDec/src/global.cpp:6-17, configfile.cpp): OriginalSequence, WZBitstream,
// KeyFrameSequence, KeyFrameInfo, RDFile, OutputSequences, FrameRate,
// ParallelMode, UseCoreNum, IntraBitstream; "-Name=Value" overrides a key.
// It reads the same inputs (WZ bitstream wzbitstream.cpp:129-210, 4:2:0 YUV
// sequences frame.cpp:70-93, key-frame information frame.cpp:197-247) and
// writes the same outputs: the RD report "<RDFile>.txt" (frame.cpp:249-337)
// and the decoded luma "<OutputSequences>.yuv" (frame.cpp:95-113).  The
// reference builds those names with sprintf into its own source buffer
// (wzbitstream.cpp:178-179), which is undefined behaviour; here they are built
// as intended.
//
// Every WZ frame of the requested range is decoded on the GPU in one
// device-resident session: the GOP recursion (DVC_Decoder.cpp:26-474) becomes
// levels of frames whose references are earlier levels' outputs.
// Skip and intra maps, intra blocks and the deblocking filter are handled as
// the reference does.  ParallelMode and UseCoreNum are read and ignored.  The per-frame
// "Decoding time" of the RD report is the session's device time divided by
// the number of WZ frames (the frames decode concurrently).
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "dvc_b200.h"

namespace {

const int kZigzag[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};  // global.cpp:36-41
const int kQTable[9][16] = {  // reconstruction.cpp:9-43
    {0},
    {16, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {32, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 0, 8, 4, 0, 0, 4, 0, 0, 0},
    {32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0, 4, 4, 0, 0},
    {64, 16, 8, 8, 16, 8, 8, 4, 8, 8, 4, 4, 8, 4, 4, 0},
    {64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 4, 8, 4, 4, 0},
    {128, 64, 32, 16, 64, 32, 16, 8, 32, 16, 8, 4, 16, 8, 4, 0}};
const int kQBits[9][16] = {  // reconstruction.cpp:44-78
    {0},
    {4, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
    {5, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 0, 3, 2, 0, 0, 2, 0, 0, 0},
    {5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0, 2, 2, 0, 0},
    {6, 4, 3, 3, 4, 3, 3, 2, 3, 3, 2, 2, 3, 2, 2, 0},
    {6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 2, 3, 2, 2, 0},
    {7, 6, 5, 4, 6, 5, 4, 3, 5, 4, 3, 2, 4, 3, 2, 0}};

[[noreturn]] void die(const std::string &msg) {
  fprintf(stderr, "dvcdec: %s\n", msg.c_str());
  exit(1);
}

const char *kKeys[] = {"OriginalSequence", "WZBitstream", "KeyFrameSequence", "KeyFrameInfo", "RDFile",
                       "OutputSequences",  "FrameRate",   "ParallelMode",     "UseCoreNum",   "IntraBitstream"};
const int kNumKeys = 10;

int key_index(const char *name) {
  for (int i = 0; i < kNumKeys; i++)
    if (strcasecmp(kKeys[i], name) == 0) return i;
  return -1;
}

struct Options {
  std::string value[kNumKeys];
  bool set_by_flag[kNumKeys] = {};
  int gpu = 0, start = -1, end = -1;
};

// configuration file: "Name = Value" triples; '#' starts a comment; values may
// be quoted (the tokenizer of configfile.cpp, which follows the H.264 JM one)
void read_config(const std::string &path, Options &o) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) die("Configure file \"" + path + "\" doesn't exist");
  std::string buf;
  char tmp[4096];
  size_t r;
  while ((r = fread(tmp, 1, sizeof tmp, f)) > 0) buf.append(tmp, r);
  fclose(f);
  std::vector<std::string> items;
  std::string cur;
  bool in_item = false, in_string = false;
  auto flush = [&]() {
    if (in_item) items.push_back(cur);
    cur.clear();
    in_item = false;
  };
  for (size_t p = 0; p < buf.size(); p++) {
    const char c = buf[p];
    if (c == '\r') continue;
    if (c == '#' && !in_string) {
      flush();
      while (p < buf.size() && buf[p] != '\n') p++;
      continue;
    }
    if (c == '\n') {
      flush();
      in_string = false;
      continue;
    }
    if ((c == ' ' || c == '\t') && !in_string) {
      flush();
      continue;
    }
    if (c == '"') {
      if (!in_string) {
        flush();
        in_item = true;
      } else {
        items.push_back(cur);
        cur.clear();
        in_item = false;
      }
      in_string = !in_string;
      continue;
    }
    in_item = true;
    cur.push_back(c);
  }
  flush();
  int count = 0;
  for (size_t i = 0; i < items.size(); i += 3) {
    if (i + 2 >= items.size()) die("Parsing error in config file: incomplete entry '" + items[i] + "'");
    const int k = key_index(items[i].c_str());
    if (k < 0) die("Parsing error in config file: Parameter Name '" + items[i] + "' not recognized.");
    if (items[i + 1] != "=") die("Parsing error in config file: '=' expected as the second token in each line.");
    if (!o.set_by_flag[k]) o.value[k] = items[i + 2];
    count++;
  }
  if (count != kNumKeys) die("Parsing error in config file: Too few parameters");
}

void parse_args(int argc, char **argv, Options &o, std::string &cfg) {
  for (int i = 1; i < argc; i++) {
    const char *a = argv[i];
    if (!strcmp(a, "-d")) {
      if (i + 1 >= argc) die("-d needs a configure file");
      cfg = argv[++i];
    } else if (!strncmp(a, "-GPUid=", 7)) {
      o.gpu = atoi(a + 7);
    } else if (!strncmp(a, "-startFrame=", 12)) {
      o.start = atoi(a + 12);
    } else if (!strncmp(a, "-endFrame=", 10)) {
      o.end = atoi(a + 10);
    } else if (a[0] == '-' && strchr(a, '=')) {
      const std::string s(a + 1);
      const size_t eq = s.find('=');
      const int k = key_index(s.substr(0, eq).c_str());
      if (k < 0) die("Invalid flag -" + s.substr(0, eq));
      o.value[k] = s.substr(eq + 1);
      o.set_by_flag[k] = true;
    } else {
      die(std::string("unknown argument ") + a +
          "\nUsage: dvcdec -d <Configure File> [-ParameterName=ParameterValue] [-GPUid=n] "
          "[-startFrame=a -endFrame=b]");
    }
  }
  if (cfg.empty()) die("Usage: dvcdec -d <Configure File> [-ParameterName=ParameterValue]");
}

struct WzFrame {
  int idx = 0, past = 0, future = 0;
  int ac_range[16] = {0};
  int skip_mode = 0, intra_mode = 0, skip_bits = 1, intra_bits = 1;
  std::vector<uint8_t> mode, crc, acc;
};

struct WzStream {
  int w = 0, h = 0, q = 0, intra_qp = 0, gop = 0, frames = 0, deblock = 0;
  std::map<int, WzFrame> wz;
};

// WZ bitstream (wzbitstream.cpp:129-210; readGOP :13-126)
WzStream read_wz(const std::string &path) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) die("File " + path + " doesn't exist");
  std::vector<uint8_t> d;
  uint8_t tmp[65536];
  size_t r;
  while ((r = fread(tmp, 1, sizeof tmp, f)) > 0) d.insert(d.end(), tmp, tmp + r);
  fclose(f);
  if (d.size() < 7) die("WZ bitstream shorter than its header");
  WzStream s;
  if (d[0] == 0) {
    s.w = 176;
    s.h = 144;
  } else if (d[0] == 1) {
    s.w = 352;
    s.h = 288;
  } else {
    die("In parsing file " + path + ": Unsupport resolution (support QCIF, CIF)");
  }
  s.q = d[1];
  if (s.q < 1 || s.q > 8) die("Qindex out of range 1..8");
  s.intra_qp = d[2];
  s.gop = d[3];
  if (s.gop < 1) die("GOP must be at least 1");
  s.frames = (d[4] << 8) | d[5];
  s.deblock = d[6];
  size_t pos = 7;
  auto take = [&](size_t k) {
    if (pos + k > d.size()) die("truncated WZ bitstream");
    const uint8_t *p = &d[pos];
    pos += k;
    return p;
  };
  const int n = s.w * s.h / 16, nb88 = s.w * s.h / 64;
  int qb = 0;
  for (int j = 0; j < 16; j++) qb += kQBits[s.q][j];
  std::vector<std::array<int, 3>> order;
  std::function<void(int, int)> rec = [&](int b, int e) {
    const int m = (b + e) / 2;
    if (m > b) {
      order.push_back({m, b, e});
      rec(b, m);
      rec(m, e);
    }
  };
  for (int i = 0; i < s.frames; i += s.gop) rec(i, std::min(i + s.gop, s.frames - 1));
  for (auto &t : order) {
    WzFrame fr;
    fr.idx = t[0];
    fr.past = t[1];
    fr.future = t[2];
    for (int j = 1; j < 16; j++) {
      const int idx = kZigzag[j];
      if (kQTable[s.q][idx] <= 0) break;
      const uint8_t *p = take(2);
      fr.ac_range[idx] = (p[0] << 8) | p[1];
    }
    fr.mode.assign(nb88, 0);
    for (int k = 0; k < 2; k++) {
      const int flag = *take(1);
      (k == 0 ? fr.skip_mode : fr.intra_mode) = flag;
      if (flag == 1) {
        // the JBIG-coded 8x8 mode map that follows a set flag (wzbitstream.cpp:38-66)
        std::vector<uint8_t> map(nb88);
        size_t used = 0;
        if (dvc_jbig_decode_mode_map(d.data() + pos, d.size() - pos, s.w / 8, s.h / 8, map.data(), &used) != DVC_OK)
          die("JBIG mode map of frame " + std::to_string(fr.idx) + " could not be decoded");
        pos += used;
        (k == 0 ? fr.skip_bits : fr.intra_bits) = (int)(used << 3) + 1;
        for (int b = 0; b < nb88; b++)
          if (map[b]) fr.mode[b] = (uint8_t)(k == 0 ? 2 : 1);
      }
    }
    fr.crc.resize(qb);
    fr.acc.resize((size_t)qb * (n / 8));
    for (int j = 0; j < qb; j++) {
      fr.crc[j] = *take(1);
      memcpy(&fr.acc[(size_t)j * (n / 8)], take(n / 8), n / 8);
    }
    s.wz[fr.idx] = std::move(fr);
  }
  return s;
}

// 4:2:0 sequence, luma of each frame (frame.cpp:70-93)
std::vector<std::vector<uint8_t>> read_sequence(const std::string &path, int frames, int w, int h) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) die("File " + path + " doesn't exist");
  const size_t fs = (size_t)w * h;
  std::vector<std::vector<uint8_t>> out(frames, std::vector<uint8_t>(fs));
  std::vector<uint8_t> uv(fs / 2);
  for (int i = 0; i < frames; i++) {
    if (fread(out[i].data(), 1, fs, f) != fs) die("Input sequence " + path + " is not enough");
    if (fread(uv.data(), 1, uv.size(), f) != uv.size() && i + 1 < frames) die("Input sequence " + path + " is not enough");
  }
  fclose(f);
  return out;
}

// key-frame bits and PSNR (frame.cpp:197-247): first "FrameNo: <i>" record
void read_frame_info(const std::string &path, int frame, int *bits, double *psnr) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) die("File " + path + " not found");
  char t[256];
  bool found = false;
  while (fscanf(f, "%255s", t) == 1) {
    if (strcmp(t, "FrameNo:") == 0 && fscanf(f, "%255s", t) == 1 && atoi(t) == frame) {
      found = true;
      break;
    }
  }
  if (!found) {
    fclose(f);
    die("In function read_one_frame_info: frame number " + std::to_string(frame) + " not found");
  }
  char v[8][256];
  for (int k = 0; k < 8; k++)
    if (fscanf(f, "%255s", v[k]) != 1) die("truncated key-frame information in " + path);
  fclose(f);
  *bits = atoi(v[1]);
  *psnr = (double)(float)atof(v[7]);
}

double frame_psnr(const uint8_t *a, const uint8_t *b, size_t n) {  // frame.cpp:115-124
  double mse = 0.0;
  for (size_t i = 0; i < n; i++) {
    const double d = (double)a[i] - (double)b[i];
    mse += d * d;
  }
  mse /= (double)n;
  return mse == 0.0 ? 0.0 : 10.0 * log10(255.0 * 255.0 / mse);
}

std::string exe_dir() {
  char buf[4096];
  const ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
  if (n <= 0) return ".";
  buf[n] = 0;
  std::string s(buf);
  return s.substr(0, s.rfind('/'));
}

}  // namespace

int main(int argc, char **argv) {
  // one hardware queue per CUDA stream (the session decodes on several); set
  // before the first CUDA call, a value from the environment wins
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  Options o;
  std::string cfg;
  parse_args(argc, argv, o, cfg);
  printf("Read configure file...\n");
  read_config(cfg, o);
  const std::string rd_file = o.value[4] + ".txt", out_file = o.value[5] + ".yuv";
  const int frame_rate = atoi(o.value[6].c_str());

  printf("Read WZ bitstream file...\n");
  WzStream s = read_wz(o.value[1]);
  const size_t fs = (size_t)s.w * s.h;
  printf("Read original sequence...\n");
  auto ori = read_sequence(o.value[0], s.frames, s.w, s.h);
  printf("Read key frame sequence...\n");
  auto recon = read_sequence(o.value[2], s.frames, s.w, s.h);
  std::vector<int> bits(s.frames, 0);
  std::vector<double> psnr(s.frames, 0.0);
  std::vector<char> is_wz(s.frames, 0);
  printf("Read key frame information...\n");
  for (int i = 0; i < s.frames; i++) read_frame_info(o.value[3], i, &bits[i], &psnr[i]);

  int start = o.start, end = o.end;
  if (start == -1 || end == -1) {
    start = 0;
    end = s.frames - 1;
  }
  if (start < 0 || end >= s.frames || start > end) die("bad -startFrame/-endFrame range");
  // WZ frames of the GOPs [i, min(i + GOP, end)] from startFrame (main.cpp:118-142)
  std::vector<int> todo;
  std::function<void(int, int)> rec = [&](int b, int e) {
    const int m = (b + e) / 2;
    if (m > b) {
      todo.push_back(m);
      rec(b, m);
      rec(m, e);
    }
  };
  for (int i = start; i <= end; i += s.gop) rec(i, std::min(i + s.gop, end));

  // intra blocks (IntraMode 1): one bitstream for the sequence, read frame by
  // frame in decoding order, frames before startFrame included (skipGOP,
  // DVC_Decoder.cpp:476-510); written over the key-frame content
  std::map<int, int> intra_bits;
  bool any_intra = false;
  for (auto &kv : s.wz) any_intra = any_intra || kv.second.intra_mode;
  if (any_intra) {
    printf("Read Intra bitstream file...\n");
    FILE *f = fopen(o.value[9].c_str(), "rb");
    if (!f) die("File " + o.value[9] + " doesn't exist");
    std::vector<uint8_t> ib;
    uint8_t tmp[65536];
    size_t r;
    while ((r = fread(tmp, 1, sizeof tmp, f)) > 0) ib.insert(ib.end(), tmp, tmp + r);
    fclose(f);
    std::vector<int> order;
    std::function<void(int, int)> walk = [&](int b, int e) {
      const int m = (b + e) / 2;
      if (m > b) {
        order.push_back(m);
        walk(b, m);
        walk(m, e);
      }
    };
    for (int i = 0; i < start; i += s.gop) walk(i, std::min(i + s.gop, end));
    for (int i = start; i <= end; i += s.gop) walk(i, std::min(i + s.gop, end));
    size_t bit = 0;
    for (int m : order) {
      const WzFrame &w = s.wz[m];
      if (!w.intra_mode) continue;
      const size_t before = bit;
      if (dvc_intra_decode_frame(ib.data(), ib.size(), &bit, s.w, s.h, s.intra_qp, w.mode.data(), recon[m].data()) !=
          DVC_OK)
        die("intra bitstream of frame " + std::to_string(m) + " could not be decoded");
      intra_bits[m] = (int)(bit - before);
    }
  }

  const std::string root = exe_dir() + "/..";
  dvc_ctx *ctx = nullptr;
  if (dvc_create((root + "/ladders").c_str(), (root + "/_tables").c_str(), o.gpu, &ctx) != DVC_OK)
    die(std::string("GPU set-up failed: ") + dvc_last_error(ctx));
  auto t0 = std::chrono::steady_clock::now();
  double device_ms = 0.0;
  std::vector<dvc_wz_frame> fr(todo.size());
  std::map<int, int> item_of;
  // each frame starts from its key-frame content with its intra blocks written in
  std::vector<std::vector<uint8_t>> outbuf;
  for (int m : todo) outbuf.push_back(recon[m]);
  for (size_t k = 0; k < todo.size(); k++) item_of[todo[k]] = (int)k;
  for (size_t k = 0; k < todo.size(); k++) {
    auto it = s.wz.find(todo[k]);
    if (it == s.wz.end()) die("frame " + std::to_string(todo[k]) + " is not in the WZ bitstream");
    const WzFrame &w = it->second;
    dvc_wz_frame &f = fr[k];
    memset(&f, 0, sizeof f);
    f.width = s.w;
    f.height = s.h;
    f.qindex = s.q;
    f.past_idx = w.past;
    f.future_idx = w.future;
    f.cur_idx = w.idx;
    // a reference that is itself decoded here is named by its output buffer
    auto ref = [&](int r) -> const uint8_t * {
      auto p = item_of.find(r);
      return p != item_of.end() && p->second < (int)k ? outbuf[p->second].data() : recon[r].data();
    };
    f.past = ref(w.past);
    f.future = ref(w.future);
    f.mode = w.mode.data();
    f.skip_mode = w.skip_mode;
    f.intra_mode = w.intra_mode;
    f.ac_range = w.ac_range;
    f.crc = w.crc.data();
    f.acc_synd = w.acc.data();
    f.recon = outbuf[k].data();
    f.deblock = s.deblock;
    f.intra_qp = s.intra_qp;
    auto pw = s.wz.find(w.past);
    f.past_mode = pw != s.wz.end() ? pw->second.mode.data() : nullptr;
  }
  if (!todo.empty()) {
    dvc_session *ses = nullptr;
    if (dvc_session_create(ctx, (int)fr.size(), fr.data(), 16, 16, &ses) != DVC_OK ||
        dvc_session_run(ses, 0, &device_ms) != DVC_OK)
      die(std::string("decode failed: ") + dvc_last_error(ctx));
    for (size_t k = 0; k < todo.size(); k++) {
      int wz_bits = 0;
      if (dvc_session_frame(ses, (int)k, recon[todo[k]].data(), &wz_bits, nullptr) != DVC_OK)
        die(std::string("result read failed: ") + dvc_last_error(ctx));
      const WzFrame &w = s.wz[todo[k]];
      bits[todo[k]] = w.skip_bits + w.intra_bits + wz_bits + (intra_bits.count(todo[k]) ? intra_bits[todo[k]] : 0);
      psnr[todo[k]] = frame_psnr(recon[todo[k]].data(), ori[todo[k]].data(), fs);
      is_wz[todo[k]] = 1;
    }
    dvc_session_destroy(ses);
  }
  const double total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  dvc_destroy(ctx);

  // RD report (frame.cpp:249-337)
  printf("output decoded RD file: %s\n", rd_file.c_str());
  FILE *rf = fopen(rd_file.c_str(), "w+");
  if (!rf) die("Could not open file: " + rd_file);
  double wz_bits = 0, key_bits = 0, wz_psnr = 0, key_psnr = 0, wz_n = 0, key_n = 0;
  const double per_frame_ms = todo.empty() ? 0.0 : device_ms / (double)todo.size();
  for (int i = start; i <= end; i++) {
    if (is_wz[i]) {
      wz_bits += bits[i];
      wz_psnr += psnr[i];
      wz_n++;
      fprintf(rf, "FrameNo: %d, Bits: %.0lf, PSNR: %.2lf (WZ), Decoding time: %.2lf ms\n", i, (double)bits[i], psnr[i],
              per_frame_ms);
    } else {
      key_bits += bits[i];
      key_psnr += psnr[i];
      key_n++;
      fprintf(rf, "FrameNo: %d, Bits: %.0lf, PSNR: %.2lf (KY)\n", i, (double)bits[i], psnr[i]);
    }
  }
  fprintf(rf, "\n");
  char text[256];
  const double avg_bits = (key_bits + wz_bits) / (key_n + wz_n) / 1000.0;
  auto both = [&](const char *t) {
    printf("%s", t);
    fprintf(rf, "%s", t);
  };
  snprintf(text, sizeof text, "File Size: %.2lf KB\n", (key_bits + wz_bits) / 8.0 / 1024.0);
  both(text);
  snprintf(text, sizeof text, "Average WZ Bits(k): %.2lf, Average WZ PSNR: %.2lf (%.0lf frames)\n",
           wz_bits / wz_n / 1000.0, wz_psnr / wz_n, wz_n);
  both(text);
  snprintf(text, sizeof text, "Average KY Bits(k): %.2lf, Average KY PSNR: %.2lf (%.0lf frames)\n",
           key_bits / key_n / 1000.0, key_psnr / key_n, key_n);
  both(text);
  snprintf(text, sizeof text, "Average Bits(k): %.2lf, Average PSNR: %.2lf (%.0lf frames)\n", avg_bits,
           (key_psnr + wz_psnr) / (key_n + wz_n), key_n + wz_n);
  both(text);
  snprintf(text, sizeof text, "BitRate (including key frame): %.2lf kbps\nTotal decoding time: %.2lf sec\n",
           avg_bits * (double)frame_rate, total_s);
  both(text);
  snprintf(text, sizeof text, "Average WZ decoding speed: %.2lf fps\n", wz_n / total_s);
  both(text);
  fclose(rf);

  // decoded luma (frame.cpp:95-113)
  printf("output decoded yuv file (only y): %s\n", out_file.c_str());
  FILE *of = fopen(out_file.c_str(), "wb+");
  if (!of) die("Could not open file: " + out_file);
  const int last = (s.frames - 1 == end) ? end : end - 1;
  for (int i = start; i <= last; i++) fwrite(recon[i].data(), 1, fs, of);
  fclose(of);
  return 0;
}
