// Entropy-coded sections on the device: every section's token stream written
// with a prebuilt ANS or prefix code, bit for bit as the reference's CPU
// writers write it, and the exact token-bit counts its rate search compares.
//
// ANS (src/codestream/ans.cpp:1700-1770, AnsReverseBits in
// src/codestream/ans_reverse_bits_internal.h): the tokens are encoded last to
// first from the state 0x13 << 16; each token pushes its hybrid-uint extra
// bits, then, when (state >> 20) >= frequency, the low 16 state bits, and the
// state becomes (state / f << 12) + reverse_map[offset + state % f]. The
// stream is the final 32-bit state followed by the pushed chunks in reverse
// push order. One CTA per section: a producer warp turns batches of tokens
// into encoder records (cluster, hybrid-uint symbol and extra bits, frequency,
// exact reciprocal, reverse-map base) while one consumer thread runs the
// state recurrence, which is serial by the format, over the previous batch
// and stores the chunks from the top of the section's slot downwards; the
// CTA then shifts the finished stream to the slot's first bit.
//
// Prefix (src/codestream/entropy.cpp:1173,2294): every token is its code
// bits followed by its extra bits, in token order; the CTA scans the token
// lengths and ORs the tokens into a shared-memory window of whole words.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "host_util.h"

namespace gjxl_b200 {
namespace {

constexpr uint32_t kAnsLogTable = 12;                 // 4096-entry tables
constexpr uint32_t kAnsTable = 1u << kAnsLogTable;
constexpr uint32_t kAnsInitialState = 0x13u << 16;    // signature << 16
constexpr uint32_t kAnsSymbols = 256;
constexpr uint32_t kPrefixSymbols = 128;
constexpr uint32_t kAnsTokenBits = 47;     // <= 31 extra bits + one 16-bit chunk
constexpr uint32_t kPrefixTokenBits = 46;  // <= 15 code bits + 31 extra bits
constexpr int kMaxCodes = 8;

// Two sections per CTA, each with three warps: one thread running the
// recurrence, a warp building encoder records and a warp placing the bits;
// both sections share the CTA's staged reverse maps.
constexpr int kAnsPairs = 2;
constexpr int kAnsThreads = 96 * kAnsPairs;
constexpr uint32_t kMaxHotClusters = 32;
constexpr int kAnsBatch = 128;    // tokens per record batch
constexpr int kPrefixThreads = 256;
constexpr int kPrefixPerThread = 4;
constexpr int kPrefixChunk = kPrefixThreads * kPrefixPerThread;
// Words a chunk can touch: its bits plus the partial word it starts in.
constexpr int kPrefixWindow = (kPrefixTokenBits * kPrefixChunk + 63) / 64 + 2;

struct Code {
  int mode;
  uint32_t context_count, cluster_count;
  const uint8_t* context_map;
  const uint8_t* uint_configs;
  const uint8_t* prefix_depths;
  const uint16_t* prefix_bits;
  const uint16_t* prefix_degenerate;
  const uint16_t* frequencies;
  const uint16_t* reverse_offsets;
  const uint16_t* reverse_map;
};

struct Tokens {
  const uint2* pairs;
  const uint32_t* values;
  const uint16_t* contexts;
  const uint32_t* offsets;
  uint32_t count;
  uint32_t capacity;  // tokens in the arrays
};

struct EmitParams {
  Code code;
  Tokens tokens;
  uint64_t* slots;        // write mode: section slots; count mode: unused
  size_t slot_capacity;   // words
  uint64_t* bit_counts;   // [section * stride + column]
  uint32_t stride, column;
  uint32_t hot_clusters;  // ANS: reverse maps staged in shared memory
  uint32_t* error;
};

__host__ __device__ __forceinline__ uint32_t TokenBits(int mode) {
  return mode == GJXL_B200_ENTROPY_ANS ? kAnsTokenBits : kPrefixTokenBits;
}

// First word of section s's slot: ceil(B * offset / 64) + 2 s.
__host__ __device__ __forceinline__ uint64_t SlotStart(uint64_t offset, uint64_t s, uint32_t b) {
  return (b * offset + 63) / 64 + 2 * s;
}

__device__ __forceinline__ void FetchToken(const Tokens& t, uint32_t i, uint32_t* context,
                                           uint32_t* value) {
  if (t.pairs != nullptr) {
    const uint2 p = t.pairs[i];
    *context = p.x;
    *value = p.y;
  } else {
    *context = t.contexts[i];
    *value = t.values[i];
  }
}

struct HybridToken {
  uint32_t symbol, extra, count;
};

// JPEG XL's hybrid-uint split of `value` under {split_exponent, msb, lsb}:
// values below 2^split are their own symbol; larger ones keep their
// exponent, `msb` bits below the leading one and the lowest `lsb` bits in
// the symbol, the rest as raw extra bits (EncodeHybridUintValidated,
// src/codestream/entropy_internal.h:31).
__device__ __forceinline__ HybridToken EncodeHybrid(uint32_t value, uint32_t split,
                                                    uint32_t msb, uint32_t lsb) {
  HybridToken h;
  if (value < (1u << split)) {
    h.symbol = value;
    h.extra = 0;
    h.count = 0;
    return h;
  }
  const uint32_t exponent = 31u - static_cast<uint32_t>(__clz(value));
  const uint32_t mantissa = value - (1u << exponent);
  h.symbol = (1u << split) + ((exponent - split) << (msb + lsb)) +
             ((mantissa >> (exponent - msb)) << lsb) + (mantissa & ((1u << lsb) - 1u));
  h.count = exponent - msb - lsb;
  h.extra = static_cast<uint32_t>((value >> lsb) & ((1ull << h.count) - 1ull));
  return h;
}

// The cluster and hybrid-uint token of one stream token under `code`;
// false for a context outside the map, a cluster outside the code or an
// invalid configuration (the reference's InvalidArgument).
__device__ __forceinline__ bool ClusterToken(const Code& code, uint32_t context, uint32_t value,
                                             uint32_t* cluster, HybridToken* h) {
  if (context >= code.context_count) return false;
  *cluster = code.context_map[context];
  if (*cluster >= code.cluster_count) return false;
  const uint8_t* config = code.uint_configs + 3 * *cluster;
  const uint32_t split = config[0], msb = config[1], lsb = config[2];
  if (split > 15 || msb > split || lsb > split - msb) return false;
  *h = EncodeHybrid(value, split, msb, lsb);
  return true;
}

// Section bounds with the checks every kernel makes: false (and the error
// bit) for decreasing offsets, tokens past the arrays' capacity or a slot
// beyond the buffer.
__device__ __forceinline__ bool SectionBounds(const EmitParams& p, uint32_t s, bool write,
                                              uint32_t* begin, uint32_t* end,
                                              uint64_t* slot_begin, uint64_t* slot_end,
                                              bool report) {
  *begin = p.tokens.offsets[s];
  *end = p.tokens.offsets[s + 1];
  const uint32_t b = TokenBits(p.code.mode);
  *slot_begin = SlotStart(*begin, s, b);
  *slot_end = SlotStart(*end, s + 1, b);
  const bool ok = *end >= *begin && *end <= p.tokens.capacity &&
                  (!write || *slot_end <= p.slot_capacity);
  if (!ok && report) {
    RaiseError(p.error, kErrorRange);
    p.bit_counts[static_cast<size_t>(s) * p.stride + p.column] = 0;
  }
  return ok;
}

// ---------------------------------------------------------------- ANS ----

// Encoder record of one token for the recurrence: {reciprocal low word,
// reciprocal high bits, frequency, reverse-map index base | staged << 31},
// and for the emitter {extra bits, extra-bit count}. A staged cluster's base
// indexes the shared-memory copy of its reverse map (slot_of != 0xFF).
__device__ __forceinline__ void AnsRecord(const Code& code, const uint8_t* slot_of,
                                          uint32_t context, uint32_t value, uint4* record,
                                          uint2* extra, bool* bad) {
  uint32_t cluster;
  HybridToken h;
  if (ClusterToken(code, context, value, &cluster, &h) && h.symbol < kAnsSymbols) {
    const uint32_t k = cluster * kAnsSymbols + h.symbol;
    const uint32_t f = code.frequencies[k];
    const uint32_t offset = code.reverse_offsets[k];
    if (f != 0 && offset + f <= kAnsTable) {
      // ceil(2^44 / f): the state stays below f * 2^20, so the high bits of
      // state * reciprocal are the exact quotient state / f.
      const uint64_t reciprocal = ((1ull << 44) + f - 1) / f;
      const uint32_t slot = slot_of[cluster];
      const uint32_t base = slot != 0xFFu ? (slot * kAnsTable + offset) | 0x80000000u
                                          : cluster * kAnsTable + offset;
      *record = make_uint4(static_cast<uint32_t>(reciprocal),
                           static_cast<uint32_t>(reciprocal >> 32), f, base);
      *extra = make_uint2(h.extra, h.count);
      return;
    }
  }
  *bad = true;
  // A harmless stand-in: frequency 4096 (reciprocal 2^32) in cluster 0.
  *record = make_uint4(0u, 1u, kAnsTable, 0u);
  *extra = make_uint2(0u, 0u);
}

// Named barriers 1 and 2: the three warps of one section.
__device__ __forceinline__ void SectionBarrier(int section) {
  if (section == 0) {
    asm volatile("bar.sync 1, 96;" ::: "memory");
  } else {
    asm volatile("bar.sync 2, 96;" ::: "memory");
  }
}

constexpr int kAnsWindow = (kAnsTokenBits * kAnsBatch + 63) / 64 + 2;

// Per-section pipeline buffers: batch k's records are filled in phase k - 1,
// consumed by the recurrence in phase k and emitted in phase k + 1.
struct AnsStage {
  uint4 records[3][kAnsBatch];
  uint2 extra[3][kAnsBatch];
  uint32_t chunks[3][kAnsBatch];  // 0x10000 | low state bits when renormalised
  unsigned long long window[kAnsWindow];
  uint32_t bad_token;
  uint32_t final_state;
  uint64_t stream_start, stream_bits;
};

// The emitter warp places one batch's bits below `*top` (the stream is
// built from its end): token i's bits, its renormalisation chunk and then
// its extra bits, start at top - L + (bits of tokens before i in the
// batch). Whole words go to the slot; the lowest, partial one is carried.
template <bool kCount>
__device__ __forceinline__ void EmitBatch(AnsStage& st, int buffer, int count, int lane,
                                          uint64_t* slots, uint64_t* top, uint64_t* carry,
                                          bool flush, uint32_t final_state) {
  uint64_t value[4];
  uint32_t length[4];
  uint32_t mine = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = 4 * lane + k;
    value[k] = 0;
    length[k] = 0;
    if (flush) {
      if (lane == 0 && k == 0) {
        value[0] = final_state;
        length[0] = 32;
      }
    } else if (i < count) {
      const uint32_t chunk = st.chunks[buffer][i];
      const uint2 e = st.extra[buffer][i];
      const uint32_t renorm = chunk >> 16;
      value[k] = (chunk & 0xFFFFu) | (static_cast<uint64_t>(e.x) << (renorm ? 16 : 0));
      length[k] = (renorm ? 16u : 0u) + e.y;
    }
    mine += length[k];
  }
  uint32_t inclusive = mine;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
    if (lane >= d) inclusive += v;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, inclusive, 31);
  if (kCount || (total == 0 && !flush)) {
    *top -= total;
    return;
  }
  const uint64_t base = *top - total;
  const uint64_t low_word = base >> 6;
  const int highest = static_cast<int>(((*top - 1) >> 6) - low_word);
  for (int j = lane; j <= highest; j += 32) {
    st.window[j] = j == highest ? *carry : 0ull;
  }
  __syncwarp();
  uint64_t at = base + (inclusive - mine);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (length[k] != 0) {
      const int j = static_cast<int>((at >> 6) - low_word);
      const int shift = static_cast<int>(at & 63);
      atomicOr(&st.window[j], static_cast<unsigned long long>(value[k] << shift));
      if (shift + static_cast<int>(length[k]) > 64) {
        atomicOr(&st.window[j + 1], static_cast<unsigned long long>(value[k] >> (64 - shift)));
      }
      at += length[k];
    }
  }
  __syncwarp();
  const int first = (flush || (base & 63) == 0) ? 0 : 1;
  for (int j = first + lane; j <= highest; j += 32) slots[low_word + j] = st.window[j];
  *carry = (base & 63) != 0 ? st.window[0] : 0ull;
  *top = base;
  __syncwarp();
}

template <bool kCount>
__global__ void __launch_bounds__(kAnsThreads) AnsSectionKernel(const __grid_constant__ EmitParams p) {
  static_assert(kAnsPairs == 2, "one named barrier per section");
  __shared__ AnsStage stage[kAnsPairs];
  __shared__ uint32_t cluster_tokens[256];
  __shared__ uint8_t slot_of[256];
  __shared__ uint8_t slot_cluster[kMaxHotClusters];
  extern __shared__ uint4 hot_storage[];  // hot_clusters reverse maps
  const uint16_t* hot_maps = reinterpret_cast<const uint16_t*>(hot_storage);
  const Code& code = p.code;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int section = warp / 3;           // warps 3 section + {0 recurrence, 1 records, 2 bits}
  const int role = warp % 3;
  const int st_thread = threadIdx.x - 96 * section;
  AnsStage& st = stage[section];
  const uint32_t s = blockIdx.x * kAnsPairs + section;
  uint32_t begin = 0, end = 0;
  uint64_t slot_begin = 0, slot_end = 0;
  const bool active = s < p.tokens.count && SectionBounds(p, s, !kCount, &begin, &end,
                                                         &slot_begin, &slot_end,
                                                         st_thread == 0);
  const uint32_t n = end - begin;
  const uint32_t batches = (n + kAnsBatch - 1) / kAnsBatch;

  // The CTA's most used clusters (by token count over its sections) get
  // their reverse maps copied into shared memory, so that most lookups of
  // the serial recurrence are shared-memory loads.
  for (int c = threadIdx.x; c < 256; c += kAnsThreads) {
    cluster_tokens[c] = 0;
    slot_of[c] = 0xFF;
  }
  if (st_thread == 0) st.bad_token = 0;
  const uint32_t hot = min(p.hot_clusters, code.cluster_count);
  if (hot > 0) {
    __syncthreads();
    if (active) {
      for (uint32_t t = begin + st_thread; t < end; t += 96) {
        uint32_t context, value;
        FetchToken(p.tokens, t, &context, &value);
        if (context < code.context_count) {
          const uint32_t cluster = code.context_map[context];
          if (cluster < code.cluster_count) atomicAdd(&cluster_tokens[cluster], 1u);
        }
      }
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < code.cluster_count; c += kAnsThreads) {
      const uint32_t mine = cluster_tokens[c];
      uint32_t rank = 0;
      for (uint32_t o = 0; o < code.cluster_count; ++o) {
        const uint32_t other = cluster_tokens[o];
        rank += other > mine || (other == mine && o < c);
      }
      if (rank < hot && mine != 0) {
        slot_of[c] = static_cast<uint8_t>(rank);
        slot_cluster[rank] = static_cast<uint8_t>(c);
      } else if (rank < hot) {
        slot_cluster[rank] = 0xFF;
      }
    }
    __syncthreads();
    constexpr uint32_t kVectors = kAnsTable * 2 / 16;  // uint4 per map
    const uint4* maps = reinterpret_cast<const uint4*>(code.reverse_map);
    for (uint32_t i = threadIdx.x; i < hot * kVectors; i += kAnsThreads) {
      const uint32_t cluster = slot_cluster[i / kVectors];
      if (cluster != 0xFFu) hot_storage[i] = maps[cluster * kVectors + i % kVectors];
    }
  }
  __syncthreads();
  if (!active) return;  // past the last CTA-wide barrier

  // Batch k (processing order) holds tokens [begin + (batches - 1 - k) *
  // kAnsBatch, ...): the last batch first.
  const auto batch_first = [&](uint32_t k) { return begin + (batches - 1 - k) * kAnsBatch; };
  const auto batch_count = [&](uint32_t k) {
    return static_cast<int>(min(static_cast<uint32_t>(kAnsBatch), end - batch_first(k)));
  };
  const auto fill = [&](uint32_t k) {
    const uint32_t first = batch_first(k);
    const int count = batch_count(k);
    const int buffer = k % 3;
    bool bad = false;
#pragma unroll 4
    for (int i = lane; i < count; i += 32) {
      uint32_t context, value;
      FetchToken(p.tokens, first + i, &context, &value);
      AnsRecord(code, slot_of, context, value, &st.records[buffer][i], &st.extra[buffer][i],
                &bad);
    }
    if (bad) st.bad_token = 1;
  };

  uint32_t state = kAnsInitialState;
  uint32_t map_bits = 0;
  uint64_t top = slot_end * 64, carry = 0;
  if (role == 1 && batches > 0) fill(0);
  SectionBarrier(section);
  for (uint32_t k = 0; k <= batches; ++k) {
    if (role == 1) {
      if (k + 1 < batches) fill(k + 1);
    } else if (role == 0) {
      if (k < batches && lane == 0) {
        const int buffer = k % 3;
        const uint4* records = st.records[buffer];
        uint32_t* chunks = st.chunks[buffer];
        const int count = batch_count(k);
        uint4 next = records[count - 1];
        for (int i = count - 1; i >= 0; --i) {
          const uint4 r = next;
          next = records[max(i - 1, 0)];
          const bool renorm = (state >> (32 - kAnsLogTable)) >= r.z;
          chunks[i] = renorm ? 0x10000u | (state & 0xFFFFu) : 0u;
          state = renorm ? state >> 16 : state;
          const uint32_t q = static_cast<uint32_t>(
            (static_cast<uint64_t>(state) * r.y + __umulhi(state, r.x)) >> 12);
          const uint32_t index = (r.w & 0x7FFFFFFFu) + (state - q * r.z);
          const uint32_t m = static_cast<int32_t>(r.w) < 0
                               ? static_cast<uint32_t>(hot_maps[index])
                               : static_cast<uint32_t>(__ldg(code.reverse_map + index));
          map_bits |= m;
          state = (q << kAnsLogTable) + m;
        }
      }
    } else if (k >= 1) {
      EmitBatch<kCount>(st, (k - 1) % 3, batch_count(k - 1), lane, p.slots, &top, &carry,
                        false, 0u);
    }
    SectionBarrier(section);
  }
  if (role == 0 && lane == 0) {
    st.final_state = state;
    if (st.bad_token != 0 || (map_bits >> kAnsLogTable) != 0) RaiseError(p.error, kErrorRange);
  }
  SectionBarrier(section);
  if (role == 2) {
    // The final state opens the stream: its 32 bits go below everything.
    EmitBatch<kCount>(st, 0, 0, lane, p.slots, &top, &carry, true, st.final_state);
    if (lane == 0) {
      if (kCount) {
        p.bit_counts[static_cast<size_t>(s) * p.stride + p.column] = slot_end * 64 - top;
      } else {
        st.stream_start = top - slot_begin * 64;
        st.stream_bits = slot_end * 64 - top;
        p.bit_counts[static_cast<size_t>(s) * p.stride + p.column] = st.stream_bits;
      }
    }
  }
  if (kCount) return;
  SectionBarrier(section);
  // Shift the stream down to the slot's first bit, 96 words at a time; every
  // word is read (at or above its destination) before any is written.
  uint64_t* slot = p.slots + slot_begin;
  const uint64_t slot_words = slot_end - slot_begin;
  const uint64_t start = st.stream_start;
  const uint64_t words = (st.stream_bits + 63) / 64;
  for (uint64_t k0 = 0; k0 < words; k0 += 96) {
    const uint64_t k = k0 + st_thread;
    uint64_t v = 0;
    if (k < words) {
      const uint64_t source = start + 64 * k;
      const uint64_t sw = source >> 6;
      const int shift = static_cast<int>(source & 63);
      v = slot[sw] >> shift;
      if (shift != 0 && sw + 1 < slot_words) v |= slot[sw + 1] << (64 - shift);
    }
    SectionBarrier(section);
    if (k < words) slot[k] = v;
    SectionBarrier(section);
  }
}

// ------------------------------------------------------------- prefix ----

template <bool kCount>
__global__ void __launch_bounds__(kPrefixThreads) PrefixSectionKernel(const __grid_constant__ EmitParams p) {
  __shared__ unsigned long long window[kPrefixWindow];
  __shared__ uint32_t warp_bits[kPrefixThreads / 32];
  __shared__ uint32_t bad_token;
  uint32_t begin, end;
  uint64_t slot_begin, slot_end;
  if (!SectionBounds(p, blockIdx.x, !kCount, &begin, &end, &slot_begin, &slot_end,
                     threadIdx.x == 0)) {
    return;
  }
  const Code& code = p.code;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* slot = p.slots + slot_begin;
  if (threadIdx.x == 0) {
    bad_token = 0;
    window[0] = 0;
  }
  uint64_t position = 0;  // bits written so far
  for (uint32_t first = begin; first < end; first += kPrefixChunk) {
    uint64_t data[kPrefixPerThread];
    uint32_t length[kPrefixPerThread];
    uint32_t mine = 0;
    bool bad = false;
#pragma unroll
    for (int k = 0; k < kPrefixPerThread; ++k) {
      const uint32_t t = first + threadIdx.x * kPrefixPerThread + k;
      data[k] = 0;
      length[k] = 0;
      if (t < end) {
        uint32_t context, value, cluster;
        HybridToken h;
        FetchToken(p.tokens, t, &context, &value);
        if (ClusterToken(code, context, value, &cluster, &h) && h.symbol < kPrefixSymbols &&
            code.prefix_depths[cluster * kPrefixSymbols + h.symbol] != 0) {
          const uint32_t depth = code.prefix_degenerate[cluster] == h.symbol
                                   ? 0u
                                   : code.prefix_depths[cluster * kPrefixSymbols + h.symbol];
          data[k] = code.prefix_bits[cluster * kPrefixSymbols + h.symbol] |
                    (static_cast<uint64_t>(h.extra) << depth);
          length[k] = depth + h.count;
        } else {
          bad = true;
        }
      }
      mine += length[k];
    }
    if (bad) bad_token = 1;
    // Exclusive scan of the threads' bit counts.
    uint32_t inclusive = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
      if (lane >= d) inclusive += v;
    }
    if (lane == 31) warp_bits[warp] = inclusive;
    __syncthreads();
    uint32_t before = inclusive - mine, chunk_bits = 0;
#pragma unroll
    for (int i = 0; i < kPrefixThreads / 32; ++i) {
      const uint32_t v = warp_bits[i];
      if (i < warp) before += v;
      chunk_bits += v;
    }
    if (!kCount) {
      // window[0] holds the partial word the chunk starts in.
      const uint64_t w0 = position >> 6;
      for (int i = 1 + threadIdx.x; i < kPrefixWindow; i += kPrefixThreads) window[i] = 0;
      __syncthreads();
      uint64_t at = (position & 63) + before;
#pragma unroll
      for (int k = 0; k < kPrefixPerThread; ++k) {
        if (length[k] != 0) {
          const int shift = static_cast<int>(at & 63);
          atomicOr(&window[at >> 6], static_cast<unsigned long long>(data[k] << shift));
          if (shift + static_cast<int>(length[k]) > 64) {
            atomicOr(&window[(at >> 6) + 1],
                     static_cast<unsigned long long>(data[k] >> (64 - shift)));
          }
          at += length[k];
        }
      }
      __syncthreads();
      const uint64_t end_bit = position + chunk_bits;
      const uint64_t full = (end_bit >> 6) - w0;  // whole words finished
      for (uint64_t i = threadIdx.x; i < full; i += kPrefixThreads) slot[w0 + i] = window[i];
      __syncthreads();
      if (threadIdx.x == 0) window[0] = (end_bit & 63) != 0 ? window[full] : 0ull;
    }
    position += chunk_bits;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (!kCount && (position & 63) != 0) slot[position >> 6] = window[0];
    if (bad_token != 0) RaiseError(p.error, kErrorRange);
    p.bit_counts[static_cast<size_t>(blockIdx.x) * p.stride + p.column] = position;
  }
}

// ------------------------------------------------------------ packing ----

// byte_offsets[s] = sum over earlier sections of ceil(bits / 8); one CTA.
__global__ void __launch_bounds__(1024) SectionByteOffsetsKernel(const uint64_t* bit_counts,
                                                                 uint32_t count,
                                                                 uint64_t* byte_offsets) {
  __shared__ uint64_t warp_sums[32];
  __shared__ uint64_t carry;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t first = 0; first < count; first += 1024) {
    const uint32_t s = first + threadIdx.x;
    const uint64_t mine = s < count ? (bit_counts[s] + 7) / 8 : 0;
    uint64_t inclusive = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
      if (lane >= d) inclusive += v;
    }
    if (lane == 31) warp_sums[warp] = inclusive;
    __syncthreads();
    uint64_t before = carry + inclusive - mine, total = 0;
    for (int i = 0; i < 32; ++i) {
      if (i < warp) before += warp_sums[i];
      total += warp_sums[i];
    }
    if (s < count) byte_offsets[s] = before;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) byte_offsets[count] = carry;
}

__global__ void __launch_bounds__(256) PackSectionsKernel(const uint64_t* slots,
                                                          size_t slot_capacity,
                                                          const uint32_t* offsets, int mode,
                                                          const uint64_t* bit_counts,
                                                          const uint64_t* byte_offsets,
                                                          uint8_t* packed, size_t capacity,
                                                          uint32_t* error) {
  const uint32_t s = blockIdx.x;
  const uint64_t bytes = (bit_counts[s] + 7) / 8;
  const uint64_t at = byte_offsets[s];
  const uint64_t first = SlotStart(offsets[s], s, TokenBits(mode));
  if (at + bytes > capacity || first * 8 + bytes > slot_capacity * 8) {
    if (threadIdx.x == 0) RaiseError(error, kErrorRange);
    return;
  }
  const uint8_t* source = reinterpret_cast<const uint8_t*>(slots + first);
  for (uint64_t i = threadIdx.x; i < bytes; i += blockDim.x) packed[at + i] = source[i];
}

// ---------------------------------------------------------------- host ----

bool ValidCode(const gjxl_b200_entropy_code* c) {
  if (c == nullptr || c->context_count == 0 || c->context_count > 65536 ||
      c->cluster_count == 0 || c->cluster_count > 256 || c->context_map == nullptr ||
      c->uint_configs == nullptr) {
    return false;
  }
  if (c->mode == GJXL_B200_ENTROPY_PREFIX) {
    return c->prefix_depths != nullptr && c->prefix_bits != nullptr &&
           c->prefix_degenerate != nullptr;
  }
  if (c->mode == GJXL_B200_ENTROPY_ANS) {
    return c->ans_frequencies != nullptr && c->ans_reverse_offsets != nullptr &&
           c->ans_reverse_map != nullptr;
  }
  return false;
}

bool ValidTokens(const gjxl_b200_token_sections* t) {
  if (t == nullptr || t->offsets == nullptr || t->count == 0) return false;
  if (t->pairs != nullptr) {
    return t->values == nullptr && t->contexts == nullptr &&
           reinterpret_cast<uintptr_t>(t->pairs) % 8 == 0;
  }
  return t->values != nullptr && t->contexts != nullptr;
}

Code DeviceCode(const gjxl_b200_entropy_code& c) {
  Code d;
  d.mode = c.mode;
  d.context_count = c.context_count;
  d.cluster_count = c.cluster_count;
  d.context_map = c.context_map;
  d.uint_configs = c.uint_configs;
  d.prefix_depths = c.prefix_depths;
  d.prefix_bits = c.prefix_bits;
  d.prefix_degenerate = c.prefix_degenerate;
  d.frequencies = c.ans_frequencies;
  d.reverse_offsets = c.ans_reverse_offsets;
  d.reverse_map = c.ans_reverse_map;
  return d;
}

Tokens DeviceTokens(const gjxl_b200_token_sections& t) {
  Tokens d;
  d.pairs = reinterpret_cast<const uint2*>(t.pairs);
  d.values = t.values;
  d.contexts = t.contexts;
  d.offsets = t.offsets;
  d.count = t.count;
  d.capacity = t.capacity;
  return d;
}

struct DeviceLimits {
  int sms = 0;
  int smem_per_sm = 0;
  int smem_per_block = 0;
};

DeviceLimits Limits() {
  DeviceLimits l;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess ||
      cudaDeviceGetAttribute(&l.sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&l.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                             device) != cudaSuccess ||
      cudaDeviceGetAttribute(&l.smem_per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                             device) != cudaSuccess) {
    cudaGetLastError();
    return DeviceLimits{};
  }
  return l;
}

// Reverse maps staged per CTA: as many as fit in the shared memory one CTA
// may take while all sections still run in one wave (up to four CTAs per
// SM), at most the code's clusters. Maps must be 16-byte aligned.
uint32_t HotClusters(const EmitParams& p) {
  if (reinterpret_cast<uintptr_t>(p.code.reverse_map) % 16 != 0) return 0;
  static const DeviceLimits limits = Limits();
  if (limits.sms <= 0 || limits.smem_per_sm <= 0) return 0;
  const int ctas = static_cast<int>((p.tokens.count + kAnsPairs - 1) / kAnsPairs);
  const int per_sm = std::min(4, std::max(1, (ctas + limits.sms - 1) / limits.sms));
  constexpr int kStatic = kAnsPairs * static_cast<int>(sizeof(AnsStage)) + 256 * 4 + 256 +
                          kMaxHotClusters + 64;
  const int budget = std::min(limits.smem_per_block, limits.smem_per_sm / per_sm - 1024) -
                     kStatic;
  const int maps = budget / static_cast<int>(kAnsTable * 2);
  return static_cast<uint32_t>(std::max(0, std::min<int>(
    {maps, static_cast<int>(kMaxHotClusters), static_cast<int>(p.code.cluster_count)})));
}

template <bool kCount>
void LaunchAns(EmitParams p, cudaStream_t stream) {
  p.hot_clusters = HotClusters(p);
  const int bytes = static_cast<int>(p.hot_clusters * kAnsTable * 2);
  if (bytes > 0 &&
      cudaFuncSetAttribute(AnsSectionKernel<kCount>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes) != cudaSuccess) {
    cudaGetLastError();
    p.hot_clusters = 0;
  }
  AnsSectionKernel<kCount><<<(p.tokens.count + kAnsPairs - 1) / kAnsPairs, kAnsThreads,
                             p.hot_clusters * kAnsTable * 2, stream>>>(p);
}

template <bool kCount>
void LaunchSections(const EmitParams& p, cudaStream_t stream) {
  if (p.code.mode == GJXL_B200_ENTROPY_ANS) {
    LaunchAns<kCount>(p, stream);
  } else {
    PrefixSectionKernel<kCount><<<p.tokens.count, kPrefixThreads, 0, stream>>>(p);
  }
}

}  // namespace
}  // namespace gjxl_b200

using namespace gjxl_b200;

extern "C" size_t gjxl_b200_entropy_slot_words(int mode, size_t tokens, size_t sections) {
  if (mode != GJXL_B200_ENTROPY_ANS && mode != GJXL_B200_ENTROPY_PREFIX) return 0;
  return SlotStart(tokens, sections, TokenBits(mode));
}

extern "C" int gjxl_b200_entropy_write_sections(const gjxl_b200_entropy_code* code,
                                                const gjxl_b200_token_sections* sections,
                                                uint64_t* slot_words, size_t slot_word_capacity,
                                                uint64_t* bit_counts, uint8_t* packed,
                                                size_t packed_capacity, uint64_t* byte_offsets,
                                                uint32_t* device_error, void* stream) {
  ClearLastError();
  if (!ValidCode(code) || !ValidTokens(sections) || slot_words == nullptr ||
      bit_counts == nullptr || slot_word_capacity == 0 ||
      (packed != nullptr && (byte_offsets == nullptr || packed_capacity == 0))) {
    return SetError(GJXL_B200_INVALID_ARGUMENT, "entropy_write_sections: invalid arguments");
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  EmitParams p;
  p.code = DeviceCode(*code);
  p.tokens = DeviceTokens(*sections);
  p.slots = slot_words;
  p.slot_capacity = slot_word_capacity;
  p.bit_counts = bit_counts;
  p.stride = 1;
  p.column = 0;
  p.hot_clusters = 0;
  p.error = device_error;
  LaunchSections<false>(p, s);
  int status = CheckLaunch("entropy sections");
  if (status != GJXL_B200_OK || packed == nullptr) return status;
  SectionByteOffsetsKernel<<<1, 1024, 0, s>>>(bit_counts, sections->count, byte_offsets);
  PackSectionsKernel<<<sections->count, 256, 0, s>>>(slot_words, slot_word_capacity,
                                                     sections->offsets, code->mode,
                                                     bit_counts, byte_offsets, packed,
                                                     packed_capacity, device_error);
  return CheckLaunch("entropy section packing");
}

extern "C" int gjxl_b200_entropy_count_sections(const gjxl_b200_entropy_code* codes,
                                                uint32_t code_count,
                                                const gjxl_b200_token_sections* sections,
                                                uint64_t* bit_counts, uint32_t* device_error,
                                                void* stream) {
  ClearLastError();
  bool ok = codes != nullptr && code_count >= 1 && code_count <= kMaxCodes &&
            ValidTokens(sections) && bit_counts != nullptr;
  for (uint32_t c = 0; ok && c < code_count; ++c) ok = ValidCode(&codes[c]);
  if (!ok) return SetError(GJXL_B200_INVALID_ARGUMENT, "entropy_count_sections: invalid arguments");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (uint32_t c = 0; c < code_count; ++c) {
    EmitParams p;
    p.code = DeviceCode(codes[c]);
    p.tokens = DeviceTokens(*sections);
    p.slots = nullptr;
    p.slot_capacity = 0;
    p.bit_counts = bit_counts;
    p.stride = code_count;
    p.column = c;
    p.hot_clusters = 0;
    p.error = device_error;
    LaunchSections<true>(p, s);
    const int status = CheckLaunch("entropy section counts");
    if (status != GJXL_B200_OK) return status;
  }
  return GJXL_B200_OK;
}
