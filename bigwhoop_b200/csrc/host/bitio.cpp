// Packet-header bit I/O and tag trees.
//
// Bit writer/reader: most-significant bit first; after a 0xFF byte only seven bits are stored
// in the next byte, so a marker can never appear inside a header (bitstream.c:277-363 writer,
// :523-548 reader, :561-612 flush).  Tag trees: 4D quad trees over the codeblocks of a
// precinct with threshold-incremental coding (tagtree.c:107-445), including the reference's
// parent linking, which keeps advancing the time-axis parent pointer across levels.
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "common.hpp"

namespace bwcb {

void BitWriter::flush() {
  if (t != 8) mem.push_back(T);
}

void BitWriter::append(const RawBits &rb) {
  for (uint64_t off = 0; off < rb.n;) {
    // as many of the next bits as the current byte has room for
    const int k = (int)std::min<uint64_t>((uint64_t)t, rb.n - off);
    const uint64_t b = off & 63;
    uint64_t v = rb.words[off >> 6] << b;
    if (b + (uint64_t)k > 64) v |= rb.words[(off >> 6) + 1] >> (64 - b);
    t = (int8_t)(t - k);
    T |= (uint8_t)((uint32_t)(v >> (64 - k)) << t);
    off += (uint64_t)k;
    if (!t) {
      mem.push_back(T);
      t = (T == 0xFF) ? 7 : 8;
      T = 0;
    }
  }
}

uchar BitReader::get_bit() {
  if (!t) {
    if (L == Lmax) return 1;
    t = (T == 0xFF) ? 7 : 8;
    T = mem[L++];
  }
  t--;
  return (uchar)((T >> t) & 1);
}

uint64_t BitReader::get_symbol(uint8_t n) {
  if (n > 8) {
    error |= 2;
    return 0;
  }
  if (bytes_used() + n <= Lmax) {
    uint64_t s = 0;
    for (int i = n; i-- > 0;) s |= (uint64_t)mem[L++] << (i * 8);
    return s;
  }
  error |= 1;
  return 0;
}

void tagtree_reset(TagTree &tt) {
  // resets up to and including the first node without a parent (tagtree.c:107-124)
  for (size_t i = 0; i < tt.nodes.size(); ++i) {
    tt.nodes[i].value = 0xFFFF;
    tt.nodes[i].threshold = 0;
    if (tt.nodes[i].parent < 0) break;
  }
}

void tagtree_init(TagTree &tt, uint64_t lX, uint64_t lY, uint64_t lZ, uint64_t lT) {
  uint32_t nlX[33] = {0}, nlY[33] = {0}, nlZ[33] = {0}, nlT[33] = {0};
  uint64_t levels = 0, number = 1;
  nlX[0] = (uint32_t)lX; nlY[0] = (uint32_t)lY; nlZ[0] = (uint32_t)lZ; nlT[0] = (uint32_t)lT;
  while ((uint64_t)nlX[levels] * nlY[levels] * nlZ[levels] * nlT[levels] > 1 && levels < 31) {
    number += (uint64_t)nlX[levels] * nlY[levels] * nlZ[levels] * nlT[levels];
    nlX[levels + 1] = (nlX[levels] + 1) >> 1;
    nlY[levels + 1] = (nlY[levels] + 1) >> 1;
    nlZ[levels + 1] = (nlZ[levels] + 1) >> 1;
    nlT[levels + 1] = (nlT[levels] + 1) >> 1;
    ++levels;
  }
  tt.leaves = lX * lY * lZ * lT;
  tt.nodes.assign(number, TagNode());
  uint64_t parent_ts = 0, node = 0;
  for (uint64_t n = 0; n < levels; ++n) {
    parent_ts += (uint32_t)(nlX[n] * nlY[n] * nlZ[n] * nlT[n]);
    for (uint32_t l = 0, d = 0; l < nlT[n]; ++l, ++d) {
      if (d >> 1) {
        parent_ts += (uint64_t)nlX[n + 1] * nlY[n + 1] * nlZ[n + 1];
        d = 0;
      }
      uint64_t parent_z = parent_ts;
      for (uint32_t k = 0, c = 0; k < nlZ[n]; ++k, ++c) {
        if (c >> 1) {
          parent_z += (uint64_t)nlX[n + 1] * nlY[n + 1];
          c = 0;
        }
        uint64_t parent_y = parent_z;
        for (uint32_t j = 0, b = 0; j < nlY[n]; ++j, ++b) {
          if (b >> 1) {
            parent_y += nlX[n + 1];
            b = 0;
          }
          uint64_t parent_x = parent_y;
          for (uint32_t i = 0, a = 0; i < nlX[n]; ++i, ++a) {
            if (a >> 1) {
              parent_x++;
              a = 0;
            }
            if (parent_x >= number || node >= number) {
              // the reference would link outside its node array here; refuse the geometry
              tt.nodes.clear();
              return;
            }
            tt.nodes[node].parent = (int64_t)parent_x;
            node++;
          }
        }
      }
    }
  }
  tagtree_reset(tt);
}

void tagtree_set(TagTree &tt, uint64_t leaf, uint16_t value) {
  int64_t n = (int64_t)leaf;
  do {
    tt.nodes[n].value = value;
    n = tt.nodes[n].parent;
  } while (n >= 0 && tt.nodes[n].value > value);
}

// encode_tagtree (tagtree.c:311-373): root to leaf, each node's value coded incrementally up
// to `threshold`; only a non-estimating call records the thresholds reached.
template <class Writer, class Tree>
static void tagtree_walk(Tree &tt, Writer &bw, uint32_t threshold, uint64_t leaf, bool store) {
  int64_t branch[64];
  int nb = 0;
  int64_t n = (int64_t)leaf;
  while (tt.nodes[n].parent >= 0) {
    branch[nb++] = n;
    n = tt.nodes[n].parent;
  }
  uint32_t tmin = 0;
  for (;;) {
    auto &node = tt.nodes[n];
    uint32_t tmp = node.threshold;
    if (tmp < tmin) tmp = tmin;
    while (node.value >= tmp && tmp < threshold) {
      tmp++;
      bw.emit(node.value >= tmp ? 0 : 1);
    }
    tmin = std::min<uint32_t>(node.value, tmp);
    if constexpr (!std::is_const_v<Tree>) {
      if (store) node.threshold = (uint16_t)tmp;
    }
    if (n == (int64_t)leaf) break;
    n = branch[--nb];
  }
}

void tagtree_encode(TagTree &tt, BitWriter &bw, uint32_t threshold, uint64_t leaf,
                    uchar estimate) {
  tagtree_walk(tt, bw, threshold, leaf, !estimate);
}

void tagtree_encode_bits(TagTree &tt, RawBits &out, uint32_t threshold, uint64_t leaf,
                         uchar estimate) {
  tagtree_walk(tt, out, threshold, leaf, !estimate);
}

void tagtree_estimate(const TagTree &tt, RawBits &out, uint32_t threshold, uint64_t leaf) {
  tagtree_walk(tt, out, threshold, leaf, false);
}

// tagtree_decode(tt, br, t, leaf) for t = 1, 2, ... while it returns 1 (the packet parser's
// loop over a codeblock's missing bit planes, tier2.c), in one walk setting: a node whose
// value and whose ancestors' values are all known is left as it is by every later call, so
// each call starts below that prefix.  The same bits are read in the same order.  Returns false
// when the leaf is still unknown after the call with t = tmax.
bool tagtree_decode_until_known(TagTree &tt, BitReader &br, uint64_t leaf, uint32_t tmax) {
  int64_t branch[64];
  int nb = 0;
  int64_t n = (int64_t)leaf;
  while (n >= 0) {
    if (tt.nodes[n].value == 0xFFFF) tt.nodes[n].value = 0;
    branch[nb++] = n;
    n = tt.nodes[n].parent;
  }
  int first = nb - 1;        // highest node on the path whose value is not yet known
  uint32_t tmin_first = 0;   // what its parent hands down
  for (uint32_t t = 1;; ++t) {
    uint32_t tmin = tmin_first;
    for (int i = first; i >= 0; --i) {
      TagNode &node = tt.nodes[branch[i]];
      if (node.threshold < tmin) {
        node.value = (uint16_t)tmin;
        node.threshold = (uint16_t)tmin;
      }
      while ((node.value == node.threshold) && (node.threshold < t)) {
        node.threshold++;
        if (!br.get_bit()) node.value++;
      }
      tmin = std::min<uint32_t>(node.value, node.threshold);
    }
    while (first >= 0) {   // extend the known prefix
      const TagNode &node = tt.nodes[branch[first]];
      if (node.value >= node.threshold) break;
      tmin_first = node.value;
      --first;
    }
    if (tt.nodes[leaf].value < t) return true;
    if (t >= tmax) return false;
  }
}

uchar tagtree_decode(TagTree &tt, BitReader &br, uint32_t threshold, uint64_t leaf) {
  int64_t branch[64];
  int nb = 0;
  int64_t n = (int64_t)leaf;
  while (n >= 0) {
    if (tt.nodes[n].value == 0xFFFF) tt.nodes[n].value = 0;
    branch[nb++] = n;
    n = tt.nodes[n].parent;
  }
  uint32_t tmin = 0;
  nb--;
  n = branch[nb];
  for (;;) {
    TagNode &node = tt.nodes[n];
    if (node.threshold < tmin) {
      node.value = (uint16_t)tmin;
      node.threshold = (uint16_t)tmin;
    }
    while ((node.value == node.threshold) && (node.threshold < threshold)) {
      node.threshold++;
      if (!br.get_bit()) node.value++;
    }
    tmin = std::min<uint32_t>(node.value, node.threshold);
    if (n == (int64_t)leaf) break;
    n = branch[--nb];
  }
  return (tt.nodes[leaf].value < threshold) ? 0 : 1;
}

}  // namespace bwcb
