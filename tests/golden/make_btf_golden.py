"""Generates tests/golden/ref_btf.npz from the reference's own BTF reader.

Run where the reference sources exist (the oracle Makefile compiles them in
place into oracle/_ref/libtempest_ref.so):

    python tests/golden/make_btf_golden.py

Each case is a small factored BTF file (seeded random SVD planes; DFMF with
one plane pair per channel, FMF0 / FMF1 with channel-interleaved U rows and
one SxV; half, float and double planes; colour models 0 and 11; dynamic range
reduction; the optional header parts: cosine flag, XML, channel names,
rotations, height map) written by oracle.btf_file_bytes and loaded through the
reference's LoadBTF (src/image/btf.cc:389-1028).  Stored per case: the file's
bytes, whether LoadBTF accepted it, and for accepted files the LightsParabolic
it derived and BTFFetchSpectrum (btf.hh:498-556) of every (lv, texel).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

# a 9-direction layout: the zenith and eight directions at 40 degrees
THETA_PHI = np.stack([np.r_[0.0, np.full(8, np.radians(40.0))],
                      np.r_[0.0, np.arange(8) * np.pi / 4]], 1).astype(np.float32)
L, W, H = 9, 5, 3
N, T = L * L, W * H


def planes(rng, fmt, ks, scale=0.3):
    if fmt == "DFMF":
        return [(rng.normal(0, scale, (N, k)), rng.normal(0, scale, (T, k))) for k in ks]
    return (rng.normal(0, scale, (N * 3, ks[0])), rng.normal(0, scale, (T, ks[0])))


_PLANES = {}


def case_planes(name):
    """The SVD planes written into case `name` (after cases() ran)."""
    if not _PLANES:
        cases()
    return _PLANES[name]


def cases():
    rng = np.random.default_rng(20240611)
    out = []

    def add(name, fmt, ds, ks, cm=0, drr=0, **kw):
        p = planes(rng, fmt, ks)
        _PLANES[name] = p
        out.append((name, fmt, ds, cm, drr, O.btf_file_bytes(THETA_PHI, W, H, p, fmt=fmt, data_size=ds,
                                                              color_model=cm, drr=drr, **kw)))

    add("dfmf_half", "DFMF", 2, (7, 5, 9))
    add("dfmf_float", "DFMF", 4, (7, 5, 9))
    add("dfmf_double", "DFMF", 8, (4, 6, 3))
    add("dfmf_float_yuv", "DFMF", 4, (6, 6, 6), cm=11)
    add("dfmf_half_yuv_v4", "DFMF", 2, (8, 3, 5), cm=11, version=4, cosine_flag=0, xml=b"<btf/>")
    add("dfmf_float_rot_v2", "DFMF", 4, (5, 5, 5), version=2, rotations=np.eye(3)[None].repeat(3, 0))
    add("fmf0_float", "FMF0", 4, (6,))
    add("fmf1_half_drr", "FMF1", 2, (5,), drr=1)
    add("fmf1_float_heightmap", "FMF1", 4, (7,), drr=0, ext_version=2,
        heightmap=np.arange(6, dtype=np.uint16).reshape(2, 3), version=3, xml=b"<a/>")
    add("fmf1_double_drr", "FMF1", 8, (4,), drr=1)
    # files LoadBTF rejects
    good = O.btf_file_bytes(THETA_PHI, W, H, planes(rng, "DFMF", (4, 4, 4)), data_size=4)
    out.append(("bad_trailing_byte", "DFMF", 4, 0, 0, good + b"\0"))
    out.append(("bad_truncated", "DFMF", 4, 0, 0, good[:-10]))
    out.append(("bad_signature", "DFMF", 4, 0, 0, good[:5] + b"09FC" + good[9:]))
    p = planes(rng, "DFMF", (4, 4, 4))
    p[2] = (p[2][0], np.vstack([p[2][1], p[2][1][:1]]))   # one SxV row too many
    out.append(("bad_column_count", "DFMF", 4, 0, 0, O.btf_file_bytes(THETA_PHI, W, H, p, data_size=4)))
    u, s = planes(rng, "FMF0", (3,))
    out.append(("bad_row_count", "FMF0", 4, 0, 0,
                O.btf_file_bytes(THETA_PHI, W, H, (u[:-3], s), fmt="FMF0", data_size=4)))
    out.append(("bad_fmf1_ext_version", "FMF1", 4, 0, 0,
                O.btf_file_bytes(THETA_PHI, W, H, planes(rng, "FMF1", (3,)), fmt="FMF1", data_size=4,
                                 ext_version=3)))
    out.append(("bad_not_btf", "DFMF", 4, 0, 0, b"?" + good[1:]))
    return out


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    rec = {}
    names = []
    for name, fmt, ds, cm, drr, data in cases():
        fd, path = tempfile.mkstemp(suffix=".btf")
        os.write(fd, data)
        os.close(fd)
        try:
            handle = O.ref().ref_btf_load(path.encode())
        finally:
            os.unlink(path)
        names.append(name)
        rec[f"{name}/bytes"] = np.frombuffer(data, np.uint8)
        rec[f"{name}/meta"] = np.array([{"DFMF": 0, "FMF0": 1, "FMF1": 2}[fmt], ds, cm, drr, W, H, L], np.int64)
        rec[f"{name}/ok"] = np.array(bool(handle))
        if not handle:
            continue
        btf = O.RefBTF.__new__(O.RefBTF)
        btf.handle = handle
        dims = np.zeros(5, np.uint32)
        O.ref().ref_btf_info(handle, dims)
        btf.width, btf.height, btf.light_count, btf.tri_count, btf.edge_count = map(int, dims)
        rec[f"{name}/lights_parabolic"] = btf.mesh().lights_parabolic
        spec = np.zeros((T, N, 3), np.float32)
        for t in range(T):
            for lv in range(N):
                O.ref().ref_btf_fetch(handle, lv, t, spec[t, lv])
        rec[f"{name}/spectra"] = spec
        O.ref().ref_btf_free(handle)
    rec["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "ref_btf.npz"), **rec)
    print("wrote", len(names), "cases")


if __name__ == "__main__":
    main()
