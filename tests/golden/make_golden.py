#!/usr/bin/env python3
"""Convert the reference's golden test files into compact fixtures.

Reads the five text fixtures the reference ships (tests/{rpt02,rpt09,upt01,
upt03,uft02}.dat under the reference tree), scatters the spin-orbital tensors
into libpt spin blocks exactly as the reference's test driver does
(test.cpp:114-151 restricted, 153-315 unrestricted (T), 317-485 restricted
(fT), 487-731 unrestricted (fT)), and writes

  tests/golden/<name>.npz   arguments of the libpt call, in pt.h layout (FP64)
  tests/golden/energies.json
      e_ref            : the energy printed in the file header (8 decimals,
                         checked at 1e-8 by test.cpp:29, 990-991)
      ref_fp64/ref_fp32: the reference library itself (compiled from its own
                         sources by oracle/Makefile into oracle/_ref) run on the
                         same arrays, FP64 and *_mp, to full precision

Run in a container that has the reference tree (the GPU box does not):
    make -C oracle && python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NAMES = ["rpt02", "rpt09", "upt01", "upt03", "uft02"]


def parse(path):
    """Header fields and the list of numeric sections, in file order."""
    with open(path) as fp:
        header = fp.readline().split()
        sections, cur = [], None
        for line in fp:
            s = line.strip()
            if not s:
                continue
            if s[0].isalpha():
                cur = []
                sections.append((s.split()[0], cur))
            else:
                cur.extend(float(x) for x in s.split())
    return header, [(n, np.array(v)) for n, v in sections]


def ovvv_full(packed, o, v):
    """Spin-orbital OVVV from its b>c packed text form (test.cpp:281-292)."""
    t = np.zeros((o, v, v, v))
    it = iter(packed)
    for i in range(o):
        for a in range(v):
            for b in range(v):
                for c in range(b):
                    x = next(it)
                    t[i, a, b, c] = x
                    t[i, a, c, b] = -x
    return t


def packed_aaaa(t, o0, o1, v0, v1):
    """Same-spin OVVV block with b>c packing (test.cpp:293-297)."""
    blk = t[o0:o1, v0:v1, v0:v1, v0:v1]
    v = v1 - v0
    rows, cols = np.tril_indices(v, -1)        # b>c in row-major order
    return blk[:, :, rows, cols].reshape(-1)


def ov_blocks(x, oa, va, ob, vb):
    """alpha-alpha block then beta-beta block (test.cpp:165-206)."""
    x = x.reshape(oa + ob, va + vb)
    return np.concatenate([x[:oa, :va].ravel(), x[oa:, va:].ravel()])


def oovv_blocks(x, oa, va, ob, vb, four=True):
    o, v = oa + ob, va + vb
    x = x.reshape(o, o, v, v)
    A, B = slice(0, oa), slice(oa, o)
    a, b = slice(0, va), slice(va, v)
    blocks = [x[A, A, a, a], x[A, B, a, b]]     # test.cpp:211-220
    if four:
        blocks += [x[B, B, b, b], x[B, A, b, a]]    # test.cpp:221-230
    return np.concatenate([q.ravel() for q in blocks])


def oovo_blocks(x, oa, va, ob, vb, four=True):
    o, v = oa + ob, va + vb
    x = x.reshape(o, o, v, o)
    A, B = slice(0, oa), slice(oa, o)
    a, b = slice(0, va), slice(va, v)
    blocks = [x[A, A, a, A], x[A, B, a, B]]     # test.cpp:235-244
    if four:
        blocks += [x[B, B, b, B], x[B, A, b, A]]    # test.cpp:245-254
    return np.concatenate([q.ravel() for q in blocks])


def ovvv_blocks(packed, oa, va, ob, vb, four=True):
    o, v = oa + ob, va + vb
    t = ovvv_full(packed, o, v)
    A, B = slice(0, oa), slice(oa, o)
    a, b = slice(0, va), slice(va, v)
    blocks = [packed_aaaa(t, 0, oa, 0, va), t[A, b, a, b].ravel()]  # 293-302
    if four:
        blocks += [packed_aaaa(t, oa, o, va, v), t[B, a, b, a].ravel()]  # 303-312
    return np.concatenate(blocks)


def convert(name, path):
    header, secs = parse(path)
    kind = name[:3]
    if kind[0] == "r":
        oa, va = int(header[0]), int(header[1])
        ob, vb = oa, va
        e_ref = float(header[2])
    else:
        oa, va, ob, vb = map(int, header[:4])
        e_ref = float(header[4])
    S = dict(secs) if kind[0] == "u" else None
    out = dict(kind=kind, oa=oa, va=va, ob=ob, vb=vb, e_ref=e_ref)
    if kind == "rpt":
        # restricted fixtures hold the libpt blocks directly (test.cpp:114-151)
        names = [n for n, _ in secs]
        vals = [v for _, v in secs]
        assert names == ["d_ov_aa", "f_ov_aa", "t1_aa", "t2_aaaa", "t2_abab",
                         "i_oovo_aaaa", "i_oovo_abab", "i_oovv_aaaa",
                         "i_oovv_abab", "i_ovvv_aaaa", "i_ovvv_abab"], names
        out.update(d_ov=vals[0], f_ov=vals[1], t1=vals[2],
                   t2=np.concatenate(vals[3:5]),
                   i_oovo=np.concatenate(vals[5:7]),
                   i_oovv=np.concatenate(vals[7:9]),
                   i_ovvv=np.concatenate(vals[9:11]))
    elif kind == "upt":
        out.update(d_ov=ov_blocks(S["d_ov"], oa, va, ob, vb),
                   f_ov=ov_blocks(S["f_ov"], oa, va, ob, vb),
                   t1=ov_blocks(S["t1"], oa, va, ob, vb),
                   t2=oovv_blocks(S["t2"], oa, va, ob, vb),
                   i_oovo=oovo_blocks(S["i_oovo"], oa, va, ob, vb),
                   i_oovv=oovv_blocks(S["i_oovv"], oa, va, ob, vb),
                   i_ovvv=ovvv_blocks(S["i_ovvv"], oa, va, ob, vb))
    elif kind == "uft":
        out.update(d_ov=ov_blocks(S["d_ov"], oa, va, ob, vb),
                   f2_ov=ov_blocks(S["f2_ov"], oa, va, ob, vb),
                   l1=ov_blocks(S["l1"], oa, va, ob, vb),
                   t2=oovv_blocks(S["t2"], oa, va, ob, vb),
                   l2=oovv_blocks(S["l2"], oa, va, ob, vb),
                   i_oovv=oovv_blocks(S["i_oovv"], oa, va, ob, vb),
                   i2_t2f2_oovo=oovo_blocks(S["i2_t2f2_oovo"], oa, va, ob, vb),
                   i3_ovvv=ovvv_blocks(S["i3_ovvv"], oa, va, ob, vb),
                   i6_oovo=oovo_blocks(S["i6_oovo"], oa, va, ob, vb),
                   i7_ovvv=ovvv_blocks(S["i7_ovvv"], oa, va, ob, vb))
    else:
        raise ValueError(kind)
    return out


def main():
    # the reference checkout (whose tests/ holds the .dat fixtures): the
    # first argument, else the REFROOT environment variable
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFROOT", "")
    if not ref or not os.path.isdir(os.path.join(ref, "tests")):
        sys.exit("usage: make_golden.py <reference checkout> (or REFROOT=...)")
    from tests.golden.fixtures import reference_energy
    energies = {}
    for name in NAMES:
        case = convert(name, os.path.join(ref, "tests", name + ".dat"))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **case)
        e64 = reference_energy(case, mp=False)
        e32 = reference_energy(case, mp=True)
        energies[name] = dict(e_ref=case["e_ref"], ref_fp64=e64, ref_fp32=e32)
        print(f"{name}: header {case['e_ref']:.8f}  ref fp64 {e64:.15e}  "
              f"fp32 {e32:.15e}")
    with open(os.path.join(HERE, "energies.json"), "w") as fp:
        json.dump(energies, fp, indent=1)


if __name__ == "__main__":
    main()
