"""Writes tests/golden/*.nwbin with NWGraph's own serializer.

Run where the NWGraph sources exist (they are compiled, never copied):

    python tests/golden/make_nwbin.py [--reference PATH]   (default: $NWG_REFERENCE_ROOT, else a
    checkout named "reference" beside this repository)

A small program, compiled against the unmodified NWGraph headers and the
project's TBB-compatible shim (oracle/tbb_compat), reads MatrixMarket
fixtures of NWGraph's data/ directory with read_mm (io/mmio.hpp:199-208),
builds adjacency<0> (uint32 offsets: the 8-byte N_ field then carries a
4-byte index_t) and index_adjacency<0, uint64_t, uint32_t> (8-byte offsets),
and writes both as index_adjacency::serialize (adjacency.hpp:158-162) does:
that member is const but calls a non-const serializer and does not compile,
so the program calls its two component serializers, the reference's own, in
the same order.  It reads the 8-byte-offset files back with the reference's
deserialize() and checks the offsets survive (the 4-byte ones cannot be:
deserialize writes 8 bytes into the 4-byte N_ and corrupts the object).  The files pin
nwg_graph_read's binary reader to the reference's format.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

PROGRAM = r'''
#include <cstdio>
#include <fstream>
#include <string>
#include "nwgraph/adjacency.hpp"
#include "nwgraph/edge_list.hpp"
#include "nwgraph/io/mmio.hpp"

// index_adjacency::serialize(path) is const but calls the non-const
// indexed_struct_of_arrays::serialize, so it does not compile; write the two
// parts it writes, in its order (adjacency.hpp:158-162), with the
// reference's own serializers.
template <class G, class Soa>
void serialize_parts(G& g, const std::string& path) {
  std::ofstream out(path, std::ofstream::binary);
  static_cast<nw::graph::unipartite_graph_base&>(g).serialize(out);
  static_cast<Soa&>(g).serialize(out);
}

// Reads the file back with the reference's deserialize.  Only for 8-byte
// offsets: with a 4-byte index_t, deserialize reads 8 bytes into N_ and
// overwrites the start of the indices_ vector behind it (the N_ quirk; the
// writer likewise stores 4 bytes of that vector object after N).
template <class G, class Soa>
int roundtrip(G& g, const std::string& path, bool read_back) {
  serialize_parts<G, Soa>(g, path);
  if (!read_back) return 0;
  G back(0);
  back.deserialize(path);
  if (back.indices_.size() != g.indices_.size()) return 1;
  for (size_t i = 0; i < g.indices_.size(); ++i)
    if (back.indices_[i] != g.indices_[i]) return 1;
  return 0;
}

int main(int argc, char** argv) {
  auto aos = nw::graph::read_mm<nw::graph::directedness::directed>(std::string(argv[1]));
  auto a0  = nw::graph::adjacency<0>(aos);
  auto a64 = nw::graph::index_adjacency<0, uint64_t, uint32_t>(aos);
  using soa32 = nw::graph::indexed_struct_of_arrays<uint32_t, uint32_t>;
  using soa64 = nw::graph::indexed_struct_of_arrays<uint64_t, uint32_t>;
  int bad = roundtrip<decltype(a0), soa32>(a0, std::string(argv[2]) + ".a0.nwbin", false) +
            roundtrip<decltype(a64), soa64>(a64, std::string(argv[2]) + ".u64.nwbin", true);
  std::printf("%s: n=%zu m=%zu offsets %zu/%zu bytes\n", argv[1], a0.indices_.size() - 1,
              std::get<0>(a0.to_be_indexed_).size(), sizeof(a0.indices_[0]), sizeof(a64.indices_[0]));
  return bad;
}
'''

FIXTURES = ("karate", "bktest2", "sherman4")  # symmetric, directed, directed with 1,104 vertices


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="NWGraph source tree")
    args = ap.parse_args()
    if args.reference is None:
        sys.path.insert(0, ROOT)
        from oracle.oracle import REFERENCE_ROOT

        args.reference = REFERENCE_ROOT
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "nwbin_writer.cpp")
        exe = os.path.join(tmp, "nwbin_writer")
        open(src, "w").write(PROGRAM)
        subprocess.check_call(["g++", "-std=c++20", "-O1", "-pthread", "-Wno-deprecated-declarations",
                               "-I", os.path.join(ROOT, "oracle", "tbb_compat"),
                               "-I", os.path.join(args.reference, "include"), src, "-o", exe])
        for name in FIXTURES:
            mtx = os.path.join(args.reference, "data", name + ".mtx")
            subprocess.check_call([exe, mtx, os.path.join(HERE, name)])
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".nwbin"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    sys.exit(main())
