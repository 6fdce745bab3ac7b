// ingest.cu -- COO text parsed on the GPU, pairs written straight into device
// COO buffers for the graph builder.
//
// The reference reads the text on one host thread (src/graph.cc:82-104):
//   while (!eof) { if (fin >> u >> v) skip the rest of the line;
//                  else { clear the error; skip the rest of the line; } }
// `>>` skips any white space, newlines included, so a record whose line holds
// fewer than two numbers continues on the next line(s); a failed extraction
// (no digits, or a value above 2^32 - 1) discards the rest of the line where
// the failure happened; a leading '-' wraps modulo 2^32, as strtoul does.
// Every record therefore starts at a line start, and which line starts are
// record starts is a chain: the next record starts at the line after the one
// where this record's parse stopped.
//
// On the device:
//   1. the file is streamed into device memory in large chunks (pinned,
//      double-buffered host staging, one cudaMemcpyAsync per chunk);
//   2. line starts: each warp counts the newlines of an 8 KiB tile with
//      coalesced 16-byte loads; a scan gives every tile its first line index;
//      a second pass writes each line's start offset in order;
//   3. one thread per line parses the record that would start there: its
//      pair, whether it succeeded, and the line where the next record would
//      start (next[k] = k + 1 unless the record spilled onto later lines);
//   4. lines whose record spills are rare: they are compacted into a jump
//      list, which one thread walks in order -- a jump from a line that is
//      itself a record start hides the lines it spans -- writing +1/-1 marks
//      into a difference array; a scan of it tells every line whether a
//      record starts there (exactly the sequential chain);
//   5. record starts with a successful parse are compacted into u[], v[].
// HBM traffic is a few passes over the file bytes plus ~40 bytes per line.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "engine.h"

namespace mce {

namespace {

constexpr uint64_t kTile = 8192;           // bytes per warp tile
constexpr uint64_t kStageBytes = 64 << 20;  // pinned staging chunk
constexpr int kWarpsPerBlock = 8;

// number of '\n' bytes in a 32-bit word
__device__ __forceinline__ uint32_t newlines_in(uint32_t w) { return __popc(__vcmpeq4(w, 0x0a0a0a0au)) >> 3; }

// newlines at positions < limit in each warp's tile (limit = L - 1: a newline
// in the last byte starts no line)
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_tile_newlines(const uint4 *s, uint64_t ntiles, uint64_t limit,
                                                                          uint64_t *counts) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles;
       t += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    uint32_t n = 0;
    for (uint64_t it = 0; it < kTile / 512; it++) {
      const uint64_t off = t * kTile + it * 512 + lane * 16;
      const uint4 q = s[off / 16];
      if (off + 16 <= limit) {
        n += newlines_in(q.x) + newlines_in(q.y) + newlines_in(q.z) + newlines_in(q.w);
      } else if (off < limit) {
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
        for (int b = 0; b < 16 && off + b < limit; b++) n += ((w[b >> 2] >> (8 * (b & 3))) & 0xff) == '\n';
      }
    }
    n = __reduce_add_sync(kFull, n);
    if (lane == 0) counts[t] = n;
  }
}

// starts[0] = 0; the newline at position q < limit starts line (rank + 1) at q + 1
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_line_starts(const uint4 *s, uint64_t ntiles, uint64_t limit,
                                                                        const uint64_t *tile_first, uint64_t *starts) {
  const uint32_t lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
  for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles;
       t += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    uint64_t base = 1 + tile_first[t];
    for (uint64_t it = 0; it < kTile / 512; it++) {
      const uint64_t off = t * kTile + it * 512 + lane * 16;
      const uint4 q = s[off / 16];
      const uint32_t w[4] = {q.x, q.y, q.z, q.w};
      uint32_t mask = 0;  // bit b: byte off + b is a counted newline
#pragma unroll
      for (int b = 0; b < 16; b++)
        if (off + b < limit && ((w[b >> 2] >> (8 * (b & 3))) & 0xff) == '\n') mask |= 1u << b;
      const uint32_t n = __popc(mask);
      uint32_t incl = n;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, d);
        if (lane >= (uint32_t)d) incl += y;
      }
      uint64_t at = base + incl - n;
      while (mask) {
        const int b = __ffs(mask) - 1;
        mask &= mask - 1;
        starts[at++] = off + b + 1;
      }
      base += __shfl_sync(kFull, incl, 31);
    }
  }
}

__device__ __forceinline__ bool is_space(uint8_t c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// one `istream >> unsigned`: skip white space (counting newlines), optional
// sign, decimal digits; fails without digits or above 2^32 - 1
__device__ __forceinline__ bool extract(const uint8_t *s, uint64_t L, uint64_t &p, uint32_t &crossed, uint32_t &out) {
  while (p < L && is_space(s[p])) {
    crossed += s[p] == '\n';
    p++;
  }
  bool neg = false;
  if (p < L && (s[p] == '+' || s[p] == '-')) {
    neg = s[p] == '-';
    p++;
  }
  if (p >= L || s[p] < '0' || s[p] > '9') return false;
  uint64_t val = 0;
  bool overflow = false;
  for (; p < L && s[p] >= '0' && s[p] <= '9'; p++)
    if (!overflow) {
      val = val * 10 + (uint64_t)(s[p] - '0');
      overflow = val > 0xFFFFFFFFULL;
    }
  if (overflow) return false;
  out = neg ? (uint32_t)(0u - (uint32_t)val) : (uint32_t)val;
  return true;
}

// the record that would start at line k: pair, success, and the line where
// the next record would start (nlines: none)
__global__ void k_parse_lines(const uint8_t *s, uint64_t L, const uint64_t *starts, uint32_t nlines, uint32_t *next,
                              uint64_t *pair, uint8_t *ok) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t p = starts[k];
    uint32_t crossed = 0, a = 0, b = 0;
    const bool good = extract(s, L, p, crossed, a) && extract(s, L, p, crossed, b);
    while (p < L && s[p] != '\n') p++;
    // the newline at p ends the record's line; the next line (if any) is k + crossed + 1
    const uint64_t nx = p < L ? (uint64_t)k + crossed + 1 : nlines;
    next[k] = (uint32_t)(nx < nlines ? nx : nlines);
    pair[k] = ((uint64_t)a << 32) | b;
    ok[k] = good;
  }
}

__global__ void k_jump_flags(const uint32_t *next, uint32_t nlines, uint32_t *flag) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
       k += (uint64_t)gridDim.x * blockDim.x)
    flag[k] = next[k] > k + 1;
}

__global__ void k_compact_u32(const uint32_t *flag, const uint32_t *pos, uint64_t n, uint32_t *out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    if (flag[k]) out[pos[k]] = (uint32_t)k;
}

// Walk the spilling lines in order.  A spill from a line that is a record
// start hides the lines it spans (k + 1 .. next[k] - 1); a spill from a hidden
// line does not count.  Marks: +1 at the first hidden line, -1 after the last.
__global__ void k_resolve_jumps(const uint32_t *jumps, const uint32_t *njumps, const uint32_t *next, uint32_t nlines,
                                uint32_t *diff) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t covered_until = 0;  // lines below this are hidden
  const uint32_t nj = *njumps;
  for (uint32_t j = 0; j < nj; j++) {
    const uint32_t k = jumps[j];
    if (k < covered_until) continue;
    const uint32_t e = next[k];
    diff[k + 1] += 1u;
    diff[e] -= 1u;  // e <= nlines: diff has nlines + 1 entries
    covered_until = e;
  }
}

// take[k] = a record starts at line k (no mark covers it) and parsed
__global__ void k_take_flags(const uint32_t *diff, const uint32_t *cover_excl, const uint8_t *ok, uint32_t nlines,
                             uint32_t *take) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
       k += (uint64_t)gridDim.x * blockDim.x)
    take[k] = (cover_excl[k] + diff[k]) == 0 && ok[k];
}

__global__ void k_emit_pairs(const uint32_t *take, const uint32_t *pos, const uint64_t *pair, uint32_t nlines,
                             uint32_t *u, uint32_t *v) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
       k += (uint64_t)gridDim.x * blockDim.x)
    if (take[k]) {
      u[pos[k]] = (uint32_t)(pair[k] >> 32);
      v[pos[k]] = (uint32_t)pair[k];
    }
}

template <typename T>
struct Dev {
  T *p = nullptr;
  cudaStream_t st = nullptr;
  mce_status alloc(uint64_t n, cudaStream_t s) {
    st = s;
    if (cudaMallocAsync(&p, std::max<uint64_t>(n, 1) * sizeof(T), s) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return MCE_ERR_OUT_OF_MEMORY;
    }
    return MCE_OK;
  }
  T *release() {
    T *q = p;
    p = nullptr;
    return q;
  }
  ~Dev() {
    if (p) cudaFreeAsync(p, st);
  }
};

struct HostFile {
  FILE *f = nullptr;
  ~HostFile() {
    if (f) std::fclose(f);
  }
};

struct Pinned {
  char *p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

// the whole file into device memory, padded with zero bytes to a whole tile
mce_status upload_file(const char *path, cudaStream_t st, Dev<uint8_t> &bytes, uint64_t *len_out) {
  HostFile hf;
  hf.f = std::fopen(path, "rb");
  if (!hf.f) return MCE_ERR_IO;
  if (std::fseek(hf.f, 0, SEEK_END) != 0) return MCE_ERR_IO;
  const long len = std::ftell(hf.f);
  if (len < 0 || std::fseek(hf.f, 0, SEEK_SET) != 0) return MCE_ERR_IO;
  const uint64_t L = (uint64_t)len;
  const uint64_t padded = (L + kTile - 1) / kTile * kTile + kTile;
  MCE_TRY(bytes.alloc(padded, st));
  MCE_CUDA_TRY(cudaMemsetAsync(bytes.p + L, 0, padded - L, st));
  Pinned stage;
  const uint64_t chunk = std::min<uint64_t>(kStageBytes, std::max<uint64_t>(L, 1));
  MCE_CUDA_TRY(cudaMallocHost(&stage.p, 2 * chunk));
  cudaEvent_t done[2] = {nullptr, nullptr};
  mce_status s = MCE_OK;
  for (int i = 0; i < 2; i++)
    if (cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming) != cudaSuccess) s = MCE_ERR_CUDA;
  uint64_t off = 0;
  for (int b = 0; s == MCE_OK && off < L; b ^= 1) {
    // the staging half is reused once its previous copy has finished
    if (cudaEventSynchronize(done[b]) != cudaSuccess) {
      s = MCE_ERR_CUDA;
      break;
    }
    const uint64_t n = std::min<uint64_t>(chunk, L - off);
    char *h = stage.p + (uint64_t)b * chunk;
    if (std::fread(h, 1, n, hf.f) != n) {
      s = MCE_ERR_IO;
      break;
    }
    if (cudaMemcpyAsync(bytes.p + off, h, n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaEventRecord(done[b], st) != cudaSuccess)
      s = MCE_ERR_CUDA;
    off += n;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess && s == MCE_OK) s = MCE_ERR_CUDA;
  for (int i = 0; i < 2; i++)
    if (done[i]) cudaEventDestroy(done[i]);
  *len_out = L;
  return s;
}

}  // namespace

mce_status parse_text_device(const char *path, cudaStream_t st, uint32_t **u_out, uint32_t **v_out,
                             uint64_t *n_out) {
  *u_out = *v_out = nullptr;
  *n_out = 0;
  Dev<uint8_t> bytes;
  uint64_t L = 0;
  MCE_TRY(upload_file(path, st, bytes, &L));
  Dev<uint32_t> u, v;
  if (L == 0) {
    MCE_TRY(u.alloc(1, st));
    MCE_TRY(v.alloc(1, st));
    *u_out = u.release();
    *v_out = v.release();
    return MCE_OK;
  }
  // 2) line starts
  const uint64_t ntiles = (L + kTile - 1) / kTile;
  const uint64_t limit = L - 1;
  Dev<uint64_t> tile_n, tile_first, total;
  MCE_TRY(tile_n.alloc(ntiles, st));
  MCE_TRY(tile_first.alloc(ntiles, st));
  MCE_TRY(total.alloc(1, st));
  const uint32_t tb = 32 * kWarpsPerBlock;
  const uint32_t tgrid = grid_for(ntiles * 32, tb);
  k_tile_newlines<<<tgrid, tb, 0, st>>>((const uint4 *)bytes.p, ntiles, limit, tile_n.p);
  note_launch();
  MCE_TRY(scan_exclusive_u64(tile_n.p, tile_first.p, ntiles, total.p, st));
  uint64_t nl = 0;
  MCE_CUDA_TRY(cudaMemcpyAsync(&nl, total.p, 8, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t nlines64 = nl + 1;
  if (nlines64 >= (1ULL << 32) - 1) return MCE_ERR_TOO_LARGE;
  const uint32_t nlines = (uint32_t)nlines64;
  Dev<uint64_t> starts;
  MCE_TRY(starts.alloc(nlines, st));
  k_line_starts<<<tgrid, tb, 0, st>>>((const uint4 *)bytes.p, ntiles, limit, tile_first.p, starts.p);
  note_launch();
  // 3) the record each line would start
  Dev<uint32_t> next, flag, pos, diff, cover;
  Dev<uint64_t> pair;
  Dev<uint8_t> ok;
  MCE_TRY(next.alloc(nlines, st));
  MCE_TRY(pair.alloc(nlines, st));
  MCE_TRY(ok.alloc(nlines, st));
  k_parse_lines<<<grid_for(nlines, 256), 256, 0, st>>>(bytes.p, L, starts.p, nlines, next.p, pair.p, ok.p);
  note_launch();
  // 4) spilling records: compact, walk in order, mark hidden lines
  MCE_TRY(flag.alloc(nlines + 1, st));
  MCE_TRY(pos.alloc(nlines + 1, st));
  MCE_TRY(diff.alloc(nlines + 1, st));
  MCE_TRY(cover.alloc(nlines + 1, st));
  k_jump_flags<<<grid_for(nlines, 256), 256, 0, st>>>(next.p, nlines, flag.p);
  note_launch();
  MCE_TRY(scan_exclusive_u32(flag.p, pos.p, nlines, pos.p + nlines, st));
  Dev<uint32_t> jumps;
  MCE_TRY(jumps.alloc(nlines, st));
  k_compact_u32<<<grid_for(nlines, 256), 256, 0, st>>>(flag.p, pos.p, nlines, jumps.p);
  note_launch();
  MCE_CUDA_TRY(cudaMemsetAsync(diff.p, 0, (nlines + 1ULL) * 4, st));
  k_resolve_jumps<<<1, 1, 0, st>>>(jumps.p, pos.p + nlines, next.p, nlines, diff.p);
  note_launch();
  MCE_TRY(scan_exclusive_u32(diff.p, cover.p, nlines, nullptr, st));
  // 5) record starts that parsed -> the COO buffers
  k_take_flags<<<grid_for(nlines, 256), 256, 0, st>>>(diff.p, cover.p, ok.p, nlines, flag.p);
  note_launch();
  MCE_TRY(scan_exclusive_u32(flag.p, pos.p, nlines, pos.p + nlines, st));
  uint32_t np = 0;
  MCE_CUDA_TRY(cudaMemcpyAsync(&np, pos.p + nlines, 4, cudaMemcpyDeviceToHost, st));
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  MCE_TRY(u.alloc(np, st));
  MCE_TRY(v.alloc(np, st));
  k_emit_pairs<<<grid_for(nlines, 256), 256, 0, st>>>(flag.p, pos.p, pair.p, nlines, u.p, v.p);
  note_launch();
  MCE_CUDA_TRY(cudaGetLastError());
  MCE_CUDA_TRY(cudaStreamSynchronize(st));
  *u_out = u.release();
  *v_out = v.release();
  *n_out = np;
  return MCE_OK;
}

}  // namespace mce
