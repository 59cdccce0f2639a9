"""Generates tests/golden/ref_error.npz from the reference build: svbrdffit's
EXR map files and svbrdf-error-tool's per-texel error.

Run where the reference sources exist (oracle/_ref/libtempest_ref.so):

    python tests/golden/make_error_golden.py

* exr/<n>/... -- images of 1..4 float channels saved by the reference's
  SaveEXRImage (src/image/exr-image.cc:200-330): the file bytes and the pixels.
* error/... -- a 6x4-texel DFMF BTF of seeded synthetic texels (ring-81;
  rebuilt by error_case(), stored as its SHA-256), perturbed ground-truth maps, and for the 4x2 region at (1, 1) the error the
  tool computes (svbrdf-error-tool.cc:88-250, restated per texel in
  oracle/ref_harness.cc with the reference's own functions): pair-wise and
  max-view, luminance and per channel, sigma maps with 2 and 3 channels.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

W, H, X0, Y0, RW, RH = 6, 4, 1, 1, 4, 2
SEED = 515


def error_case():
    """The BTF bytes and the (region) maps of the error golden."""
    tp = O.ring81_angles()
    lp = O.angles_to_parabolic(tp)
    T = W * H
    truths = [O.synth_truth(SEED, 1, t) for t in range(T)]
    rgb = np.stack([O.synth_render(SEED, t, truths[t], lp) for t in range(T)])
    cols = np.array([(H - 1 - t // W) * W + t % W for t in range(T)])
    planes = []
    for c in range(3):
        S = np.zeros((T, T), np.float32)
        S[cols, np.arange(T)] = 1.0
        planes.append((rgb[:, :, c].T.astype(np.float32), S))
    data = O.btf_file_bytes(tp, W, H, planes, data_size=4)
    rng = np.random.default_rng(SEED)
    reg = [(Y0 + y) * W + X0 + x for y in range(RH) for x in range(RW)]
    t_ = [truths[i] for i in reg]
    diffuse = np.array([t.kd[:] for t in t_], np.float32) * rng.uniform(0.9, 1.1, (len(reg), 3)).astype(np.float32)
    specular = np.array([t.ks[:] for t in t_], np.float32) * rng.uniform(0.8, 1.2, (len(reg), 3)).astype(np.float32)
    sigma = np.array([t.sigma[:] for t in t_], np.float32) * rng.uniform(0.9, 1.1, (len(reg), 2)).astype(np.float32)
    basis = np.array([t.quat[:] for t in t_], np.float32)
    basis = basis + 0.02 * rng.standard_normal(basis.shape).astype(np.float32)
    basis /= np.linalg.norm(basis, axis=1, keepdims=True)
    sz = rng.uniform(0.5, 2.0, (len(reg), 1)).astype(np.float32)
    sigma3 = np.concatenate([sigma * sz, sz], 1)   # (sx sz, sy sz, sz): the tool divides by sz
    shp = lambda a: a.reshape(RH, RW, -1)
    return data, shp(diffuse), shp(specular), shp(sigma), shp(sigma3), shp(basis.astype(np.float32))


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    rec = {}
    rng = np.random.default_rng(7)
    for c in range(1, 5):
        img = rng.normal(0, 2, (5, 7, c)).astype(np.float32)
        fd, path = tempfile.mkstemp(suffix=".exr")
        os.close(fd)
        try:
            assert O.ref().ref_exr_save(path.encode(), 7, 5, c, img)
            rec[f"exr/{c}/bytes"] = np.frombuffer(open(path, "rb").read(), np.uint8)
        finally:
            os.unlink(path)
        rec[f"exr/{c}/pixels"] = img

    data, diffuse, specular, sigma, sigma3, basis = error_case()
    fd, path = tempfile.mkstemp(suffix=".btf")
    os.write(fd, data)
    os.close(fd)
    try:
        handle = O.ref().ref_btf_load(path.encode())
    finally:
        os.unlink(path)
    assert handle
    for method in (0, 1):
        for color in (0, 1):
            nch = 3 if color else 1
            rmse = np.zeros((RH, RW, nch), np.float32)
            psnr = np.zeros((RH, RW, nch), np.float32)
            for y in range(RH):
                for x in range(RW):
                    r3, p3 = np.zeros(3, np.float32), np.zeros(3, np.float32)
                    O.ref().ref_error_texel(handle, X0 + x, Y0 + y, diffuse[y, x], specular[y, x], sigma[y, x],
                                            basis[y, x], method, color, r3, p3)
                    rmse[y, x], psnr[y, x] = r3[:nch], p3[:nch]
            rec[f"error/{method}/{color}/rmse"] = rmse
            rec[f"error/{method}/{color}/psnr"] = psnr
    O.ref().ref_btf_free(handle)
    # the BTF itself is regenerated by error_case(); its digest pins it
    import hashlib

    rec["error/btf_sha256"] = np.frombuffer(hashlib.sha256(data).digest(), np.uint8)
    for k, v in (("diffuse", diffuse), ("specular", specular), ("sigma", sigma), ("sigma3", sigma3),
                 ("basis", basis)):
        rec[f"error/{k}"] = v
    rec["error/region"] = np.array([X0, Y0, RW, RH, W, H])
    np.savez_compressed(os.path.join(HERE, "ref_error.npz"), **rec)
    print("wrote", len(rec), "arrays")


if __name__ == "__main__":
    main()
