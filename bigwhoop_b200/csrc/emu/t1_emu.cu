// Host build of the tier-1 encoder's kernel bodies, for the CPU unit tests of their logic.
//
// The context-modelling body (t1_model.cuh) runs here as 256 cooperative fibers on one host
// thread -- each fiber is one thread of the CUDA block, and wherever the block calls
// __syncthreads a fiber yields; the scheduler resumes the fibers round-robin, so every fiber
// reaches a barrier before any passes it -- and the MQ lane body (t1_mq.cuh) and the coder's
// finish (t1_common.cuh) run directly.  It is the same source the CUDA kernels are compiled from.
// This library is test infrastructure: it is built as its own shared object
// (lib/emu/<precision>/libt1emu.so), is not linked into libbwc.so, and nothing in the product
// calls it.  The fiber switch is x86-64 System V code.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../kernels/t1_dec.cuh"
#include "../kernels/t1_model.cuh"
#include "../kernels/t1_mq.cuh"

// Saves the callee-saved registers on the current stack, stores the stack pointer in *from,
// switches to the stack `to` and restores what was saved there.
extern "C" void t1emu_switch(void **from, void *to);
asm(R"(
.text
.globl t1emu_switch
.type t1emu_switch,@function
t1emu_switch:
  pushq %rbp
  pushq %rbx
  pushq %r12
  pushq %r13
  pushq %r14
  pushq %r15
  movq %rsp, (%rdi)
  movq %rsi, %rsp
  popq %r15
  popq %r14
  popq %r13
  popq %r12
  popq %rbx
  popq %rbp
  ret
.size t1emu_switch, .-t1emu_switch
)");

namespace {

using namespace bwcb;
using namespace bwcb::t1;

constexpr size_t kFiberStack = 256 * 1024;

struct Fibers;
struct Fiber {
  void *sp = nullptr;
  bool done = false;
  int tid = 0;
  Fibers *owner = nullptr;
};

struct Fibers {
  void *sched_sp = nullptr;
  Fiber *current = nullptr;
  void (*body)(int tid, void *arg) = nullptr;
  void *arg = nullptr;
  std::vector<Fiber> f;
  std::vector<uint8_t *> stacks;
};

thread_local Fibers *g_fibers = nullptr;

void yield_fiber() {
  Fibers *fs = g_fibers;
  t1emu_switch(&fs->current->sp, fs->sched_sp);
}

extern "C" void t1emu_fiber_entry() {
  Fibers *fs = g_fibers;
  Fiber *me = fs->current;
  fs->body(me->tid, fs->arg);
  me->done = true;
  for (;;) t1emu_switch(&me->sp, fs->sched_sp);   // never resumed again
}

// runs body(tid, arg) for tid in [0, n) as fibers until all have returned
void run_fibers(int n, void (*body)(int, void *), void *arg) {
  Fibers fs;
  fs.body = body;
  fs.arg = arg;
  fs.f.resize(n);
  for (int i = 0; i < n; ++i) {
    uint8_t *stack = static_cast<uint8_t *>(std::aligned_alloc(64, kFiberStack));
    fs.stacks.push_back(stack);
    uintptr_t top = (reinterpret_cast<uintptr_t>(stack) + kFiberStack) & ~uintptr_t(15);
    void **sp = reinterpret_cast<void **>(top);
    *--sp = nullptr;                                            // return slot of the entry
    *--sp = reinterpret_cast<void *>(&t1emu_fiber_entry);       // popped by `ret`
    for (int r = 0; r < 6; ++r) *--sp = nullptr;                // rbp rbx r12 r13 r14 r15
    fs.f[i].sp = sp;
    fs.f[i].tid = i;
    fs.f[i].owner = &fs;
  }
  Fibers *prev = g_fibers;
  g_fibers = &fs;
  for (;;) {
    bool any = false;
    for (int i = 0; i < n; ++i) {
      if (fs.f[i].done) continue;
      any = true;
      fs.current = &fs.f[i];
      t1emu_switch(&fs.sched_sp, fs.f[i].sp);
    }
    if (!any) break;
  }
  g_fibers = prev;
  for (uint8_t *s : fs.stacks) std::free(s);
}

struct HostShared {
  uint32_t vals[kModelBlock] = {};
  int orflag[3] = {0, 0, 0};
  int or_calls[kModelBlock] = {};
};

struct HostBlock {
  int tid;
  HostShared *hs;
  void sync() { yield_fiber(); }
  // flag k = call number mod 3: set before the barrier, read after it; the flag of the call
  // before is cleared by thread 0 after the barrier and is next set after the following one
  int sync_or(int v) {
    const int k = hs->or_calls[tid]++ % 3;
    if (v) hs->orflag[k] = 1;
    sync();
    const int r = hs->orflag[k];
    if (tid == 0) hs->orflag[(k + 2) % 3] = 0;
    return r;
  }
  uint32_t scan(uint32_t v, uint32_t *total) {
    hs->vals[tid] = v;
    sync();
    uint32_t s = 0, tot = 0;
    for (int i = 0; i < kModelBlock; ++i) {
      if (i < tid) s += hs->vals[i];
      tot += hs->vals[i];
    }
    sync();
    *total = tot;
    return s;
  }
  uint32_t reduce_max(uint32_t v) {
    hs->vals[tid] = v;
    sync();
    uint32_t m = 0;
    for (int i = 0; i < kModelBlock; ++i) m = m > hs->vals[i] ? m : hs->vals[i];
    sync();
    return m;
  }
  void add(long long *p, long long v) { *p += v; }
  unsigned long long reserve(unsigned long long *c, unsigned long long n) {
    const unsigned long long b = *c;
    *c += n;
    return b;
  }
  void copy16(uint8_t *dst, const uint8_t *src, uint32_t n16) {
    for (uint32_t i = (uint32_t)tid; i < n16; i += kModelBlock) std::memcpy(dst + 16ull * i, src + 16ull * i, 16);
  }
  void or_flag(uint32_t *f, uint32_t v) { *f |= v; }
};

struct ModelJob {
  HostShared *hs;
  ModelShared *sm;
  uint8_t *stage;
  const bwc_float *work;
  const CbDev *cb;
  const SbDev *sb;
  const T1EncOut *out;
};

void model_fiber(int tid, void *arg) {
  ModelJob &j = *static_cast<ModelJob *>(arg);
  HostBlock blk{tid, j.hs};
  model_codeblock(blk, *j.sm, j.stage, j.work, *j.cb, *j.sb, *j.out, 0, &dev::h_sig2ctx[0][0],
                  dev::h_sig2xi, dev::h_xi2cont);
}

}  // namespace

extern "C" {

// Tier-1 encoding of one codeblock of `work` (dims x fastest) with the kernel bodies on the host.
//   box: X0 Y0 Z0 TS0 X1 Y1 Z1 TS1; cls: significance-context class; erres: segmentation symbols.
// Outputs: K, Z; pass_count[Z] decisions per pass; dmse[Z] distortion decreases; the decisions
// of all passes back to back in symbols (up to symbols_cap); L[Z], S[Z + 1] and the coded bytes
// (bytes_cap of room); flags as the kernels set them.  Codeblocks up to 4096 stripe columns.
// Returns the number of decisions, or -1 on bad arguments.
long long t1emu_encode(const bwc_float *work, const uint64_t *dims, const uint64_t *box,
                       bwc_float qt_eff, double gain_step2, int cls, int erres, uint8_t *K,
                       uint8_t *Z, uint32_t *pass_count, int64_t *dmse, uint8_t *symbols,
                       uint64_t symbols_cap, uint32_t *L, uint16_t *S, uint8_t *bytes,
                       uint32_t bytes_cap, uint32_t *flags) {
  CbDev cb{};
  cb.x0 = (uint32_t)box[0];
  cb.y0 = (uint32_t)box[1];
  cb.z0 = (uint32_t)box[2];
  cb.t0 = (uint32_t)box[3];
  cb.w = (uint32_t)(box[4] - box[0]);
  cb.h = (uint32_t)(box[5] - box[1]);
  cb.d = (uint32_t)(box[6] - box[2]);
  cb.nt = (uint32_t)(box[7] - box[3]);
  cb.base = 0;
  cb.sy = dims[0];
  cb.sz = dims[0] * dims[1];
  cb.st = dims[0] * dims[1] * dims[2];
  cb.out_off = 0;
  cb.out_cap = bytes_cap;
  cb.scratch_off = 0;
  const uint64_t ncols = (uint64_t)cb.w * ((cb.h + 3) / 4) * cb.d * cb.nt;
  if (!ncols || ncols > kModelMaxCols) return -1;
  SbDev sb{};
  sb.gain_step2 = gain_step2;
  sb.qt_eff = qt_eff;
  sb.cls = (uint32_t)cls;
  sb.erres = erres ? 1u : 0u;

  std::vector<uint8_t> planes(model_plane_bytes(ncols) + 64, 0);
  const uint64_t arena_cap = stream_bound(ncols, kPrecBit + 1);
  std::vector<uint8_t> arena(arena_cap + 256, 0);
  unsigned long long used[2] = {0, 0};   // arena bytes reserved, decisions coded
  std::vector<uint64_t> snaps(2 * kMaxPasses + 16, 0);
  std::vector<int64_t> dm(kMaxPasses, 0);
  std::vector<uint32_t> pc(kMaxPasses, 0);
  std::vector<uint64_t> po(kMaxPasses, 0);
  uint32_t slopes[2] = {0xFFFF, 0};
  uint32_t fl = 0;
  T1EncOut o;
  o.bytes = bytes;
  o.K = K;
  o.Z = Z;
  o.L = L;
  o.S = S;
  o.slopes = slopes;
  o.flags = &fl;
  o.planes = planes.data();
  o.snaps = snaps.data();
  o.dmse = dm.data();
  o.symbols = arena.data();
  o.sym_cap = arena_cap;
  o.sym_used = used;
  o.pass_count = pc.data();
  o.pass_off = po.data();

  std::vector<uint8_t> smem(sizeof(ModelShared) + kStageBytes + 64, 0);
  ModelShared &sm = *reinterpret_cast<ModelShared *>(smem.data());
  uint8_t *stage = smem.data() + ((sizeof(ModelShared) + 15) & ~size_t(15));
  HostShared hs;
  ModelJob job{&hs, &sm, stage, work, &cb, &sb, &o};
  run_fibers(kModelBlock, model_fiber, &job);
  const int z = *Z;
  long long total = 0;
  for (int p = 0; p < z; ++p) {
    pass_count[p] = pc[p];
    dmse[p] = dm[p];
    for (uint32_t i = 0; i < pc[p]; ++i) {
      if ((uint64_t)total < symbols_cap) symbols[total] = arena[po[p] + i];
      ++total;
    }
  }
  if (*K && !(fl & 8u)) {
    MqState e{0x8000u, 0u, 0u, 12, -1};
    ByteSink bo{bytes, bytes_cap, 0u};
    uint32_t slot[dev::kCtxTotal];
    mq_code_stream(e, bo, arena.data() + po[0], pc.data(), z, dev::h_mq_states, slot, 1,
                   snaps.data());
    uint32_t smin, smax;
    t1_finish(e, bo, *K, z, snaps.data(), dm.data(), gain_step2, L, S, &smin, &smax);
    fl |= bo.flags;
  }
  *flags = fl;
  return total;
}

// Tier-1 decoding of one codeblock with the decoder's kernel bodies on the host: Z passes of
// `len` coded bytes into the zeroed working buffer `work` (dims x fastest), as bwc_decompress's
// decode stage.  Codeblocks up to 4096 stripe columns.  Returns 0, or -1 on bad arguments.
int t1emu_decode(bwc_float *work, const uint64_t *dims, const uint64_t *box, bwc_float qt_eff,
                 int cls, int erres, int K, int Z, const uint8_t *bytes, uint32_t len) {
  CbDev cb{};
  cb.x0 = (uint32_t)box[0];
  cb.y0 = (uint32_t)box[1];
  cb.z0 = (uint32_t)box[2];
  cb.t0 = (uint32_t)box[3];
  cb.w = (uint32_t)(box[4] - box[0]);
  cb.h = (uint32_t)(box[5] - box[1]);
  cb.d = (uint32_t)(box[6] - box[2]);
  cb.nt = (uint32_t)(box[7] - box[3]);
  cb.base = 0;
  cb.sy = dims[0];
  cb.sz = dims[0] * dims[1];
  cb.st = dims[0] * dims[1] * dims[2];
  const uint32_t ncols = cb.w * ((cb.h + 3) / 4) * cb.d * cb.nt;
  if (!ncols || ncols > kModelMaxCols) return -1;
  const int ngroups = (int)((ncols + 15) / 16);
  // the coded bytes, 16-byte aligned with zero padding after them
  std::vector<uint8_t> hold((size_t)len + 96, 0);
  uint8_t *data = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(hold.data()) + 15) & ~uintptr_t(15));
  if (len) std::memcpy(data, bytes, len);
  std::vector<u64> sig(ngroups), sgn(ngroups), pi(ngroups), del(ngroups), bits(ngroups);
  std::vector<u64> planes((size_t)ngroups * (kPrecBit + 1), 0);
  uint32_t slot[dev::kCtxTotal];
  static DecTables tabs;
  for (int i = 0; i < 256; ++i) dec_table_entry(tabs, i, &dev::h_sig2ctx[0][0], dev::h_sig2xi, dev::h_xi2cont);
  const DecOut res = decode_seq(data, len, K, Z, erres != 0, cb.w, cb.h, ncols, cls, sig.data(),
                                sgn.data(), pi.data(), del.data(), bits.data(), slot,
                                dev::h_mq_states, tabs, planes.data());
  for (int g = 0; g < ngroups; ++g)
    dequant_group(g, ngroups, K, res, planes.data(), sgn[g], pi[g], cb, qt_eff, work, cb.w, cb.h,
                  ncols);
  return 0;
}

// MQ coding, truncation lengths and slopes of one codeblock's decisions (back to back, as
// t1emu_encode returns them, pass_count[Z] per pass) with the coder in two halves: the interval
// half codes every chunk into (add, shift) pairs first, the register half then applies them, as
// the split MQ kernel's two warps do chunk by chunk.  Outputs L[Z], S[Z + 1], the bytes
// (bytes_cap of room) and flags.  Returns 0, or -1 on bad arguments.
int t1emu_mq_split(const uint8_t *symbols, const uint32_t *pass_count, int K, int Z,
                   const int64_t *dmse, double gain_step2, uint32_t *L, uint16_t *S,
                   uint8_t *bytes, uint32_t bytes_cap, uint32_t *flags) {
  if (Z < 0 || Z > kMaxPasses) return -1;
  // the arena layout: every pass starts on a 16-byte boundary, readable 32 bytes past the end
  std::vector<uint64_t> start(Z + 1, 0);
  uint64_t pos = 0, src = 0;
  for (int p = 0; p < Z; ++p) {
    start[p] = pos;
    pos += ((uint64_t)pass_count[p] + 15) & ~15ull;
  }
  std::vector<uint8_t> arena(pos + 64, 0);
  for (int p = 0; p < Z; ++p) {
    if (pass_count[p]) std::memcpy(arena.data() + start[p], symbols + src, pass_count[p]);
    src += pass_count[p];
  }
  const uint32_t nchunks = stream_chunks(pass_count, Z);
  std::vector<uint32_t> pairs((size_t)nchunks * 16 + 16, 0);
  std::vector<uint16_t> snapA(kMaxPasses, 0);
  std::vector<uint64_t> snaps(2 * kMaxPasses + 16, 0);
  MqSlot slot[dev::kCtxTotal];
  MqProducer P;
  mq_producer_init(P, arena.data(), pass_count, Z, dev::h_mq_states, slot, 1);
  for (uint32_t k = 0; k < nchunks; ++k)
    if (!mq_produce_chunk(P, pairs.data() + (size_t)k * 16, 1, snapA.data(), 1)) return -1;
  mq_producer_passes(P, snapA.data(), 1);
  MqConsumer Q;
  mq_consumer_init(Q, pass_count, Z, bytes, bytes_cap);
  for (uint32_t k = 0; k < nchunks; ++k)
    if (!mq_consume_chunk(Q, pairs.data() + (size_t)k * 16, 1, snaps.data())) return -1;
  mq_consumer_passes(Q, snaps.data());
  mq_consumer_overflow(Q);
  for (int p = 0; p < Z; ++p) snaps[2 * p] |= (uint64_t)snapA[p] << 48;
  uint32_t smin, smax;
  t1_finish(Q.e, Q.bo, K, Z, snaps.data(), dmse, gain_step2, L, S, &smin, &smax);
  *flags = Q.bo.flags;
  return 0;
}

// 8x8 bit transpose as the kernels use it (for its unit test)
unsigned long long t1emu_transpose8(unsigned long long x) { return transpose8(x); }

}  // extern "C"
