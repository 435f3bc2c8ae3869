"""Generates tests/golden/*.npz from the reference's own code.

Runs the reference's common/ covariance code (Tomo_struct + matcov_tile,
compiled from the reference sources by ``make -C oracle ref`` into
oracle/_ref/libmoao_ref.so) on the test systems and stores, per system:
the geometry tables, 3000 seeded sample elements of each of Cmm (lower),
Ctm and Ctt, and size-independent checksums of the full matrices.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(HERE)]

import oracle as O  # noqa: E402
import systems  # noqa: E402

TABLES = ["u", "v", "X", "Y", "sspSizeL", "L0diff", "cn2", "Nsubap", "Nssp", "noiseNGS",
          "noiseLGSxx", "noiseLGSyy", "noiseLGSxy", "alphaX", "alphaY", "lgsExt", "lgsTheta", "mr"]
NSAMPLE = 3000


def samples(rng, nr, nc, lower):
    r = rng.integers(0, nr, NSAMPLE)
    c = rng.integers(0, nc, NSAMPLE)
    if lower:
        r, c = np.maximum(r, c), np.minimum(r, c)
    return r, c


def main(names=("small", "check2", "check10")):
    if not O.RefTomo.available():
        raise SystemExit("oracle/_ref/libmoao_ref.so missing: run `make -C oracle ref`")
    for name in names:
        sf, af = systems.files(name)
        t = O.RefTomo(sf, af)
        info = t.info
        out = {k: t.table(k) for k in TABLES}
        nm, nts = info.nmeas, info.nmeasts
        rng = np.random.default_rng(20261203)
        for tag, typ, nr, nc in (("Cmm", 1, nm, nm), ("Ctm", 3, nts, nm), ("Ctt", 4, nts, nts)):
            if typ == 3:
                t.setTarget(0)
            M = t.matcov_full(nr, nc, typ, nthreads=os.cpu_count() or 1)
            r, c = samples(rng, nr, nc, typ == 1)
            out[f"{tag}_rows"], out[f"{tag}_cols"], out[f"{tag}_vals"] = r, c, M[r, c]
            part = np.tril(M) if typ == 1 else M
            out[f"{tag}_sum"] = np.array(part.sum())
            out[f"{tag}_fro"] = np.array(np.linalg.norm(part))
            out[f"{tag}_colsum"] = part.sum(axis=0)
        out["info"] = np.array([info.nW, info.nLgs, info.nLayer, info.Nx, nm, nts])
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
