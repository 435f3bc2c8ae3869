"""Generates the check-set fixtures from the reference tree (run where it exists).

1. ``check_sets.json``: the six systems of the reference's ``datafile/check``
   directory (nx456, nx5120 and nx10112 subapertures, 2 and 10 layers), parsed
   positionally the way ``SysParams::getParams`` (common/tomo_struct/
   sysParams.cpp:166-204) and ``AtmParams::getParams`` (common/tomo_struct/
   atmParams.cpp:93-102) read them: one comment line, then one value line, per
   field. The tests write them back in the same format (moao_b200.params).
2. ``ref_<set>.npz`` per check set and ``ref_elt.npz`` for the seeded ELT-scale
   system (39 m, 64x64, 6 LGS + 2 NGS + truth sensor, 35 layers): outputs of the
   reference's own Tomo_struct and matcov_tile (oracle/_ref/libmoao_ref.so,
   compiled unchanged from the reference sources by ``make -C oracle ref``):
   the geometry tables (large ones as seeded samples plus checksums) and
   48x48 tiles of Cmm (type 1), Ctm (type 3) and Ctt (type 4) at fixed and
   seeded offsets. ELT tiles are placed on every kind of WFS pair the
   covariance kernels treat differently (LGS x LGS offset tables, NGS x LGS and
   truth sensor x LGS shared-point blocks, NGS x NGS, diagonal blocks, the x/y
   boundaries inside a WFS, the last rows).

3. ``legacy_sets.json``: the ten legacy-layout system files of the reference's
   ``datafile/benchmark`` directory (22 fields: diam, obs, nW, Nssp, gsAlt, type,
   nLgs, alphaX, alphaY, XPup, YPup, thetaML, thetaCam, sensibilite, tracking,
   pasDphi, ncpu, lgs_cst, noise_var, spot_width, lgs_alt, lgs_depth), value
   lines as numbers. (The benchmark profiles are not kept: they declare 61
   layers and list 60 altitudes, which the reference's reader rejects.)

    REF=/root/reference python tests/golden/make_check_sets.py
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from moao_b200 import params as P  # noqa: E402

SETS = ["nx456_nLayers2_wfs6_Nssp10", "nx456_nLayers10_wfs6_Nssp10",
        "nx5120_nLayers2_wfs8_Nssp29", "nx5120_nLayers10_wfs8_Nssp29",
        "nx10112_nLayers2_wfs8_Nssp41", "nx10112_nLayers10_wfs8_Nssp41"]
SMALL_TABLES = ["sspSizeL", "L0diff", "cn2", "Nsubap", "Nssp", "noiseNGS", "alphaX", "alphaY",
                "lgsExt", "lgsTheta", "mr"]
LARGE_TABLES = ["u", "v", "X", "Y", "noiseLGSxx", "noiseLGSyy", "noiseLGSxy"]
TILE = 48


def read_positional(path):
    """Value lines of a reference parameter file (every second line, from the second)."""
    lines = open(path).read().splitlines()
    return [lines[i].split() for i in range(1, len(lines), 2)]


def parse_sys(path):
    vals = read_positional(path)
    fields = [f for f, _ in P._SYS_COMMENTS]
    s = P.SysParams()
    ints = {"nW", "nLgs", "nTarget", "nssp", "ncpu", "RON"}
    for f, v in zip(fields, vals):
        cur = getattr(s, f)
        if isinstance(cur, list):
            conv = int if f == "gsType" else float
            setattr(s, f, [conv(float(x)) for x in v])
        elif f in ints:
            setattr(s, f, int(float(v[0])))
        else:
            setattr(s, f, float(v[0]))
    return s


def parse_atm(path):
    vals = read_positional(path)
    n = int(float(vals[0][0]))
    return P.AtmParams(nLayer=n, r0=float(vals[1][0]), cn2=[float(x) for x in vals[2][:n]],
                       h=[float(x) for x in vals[3][:n]], L0=[float(x) for x in vals[4][:n]])


def tiles_for(nm, nts, rng, extra):
    """(type, row0, col0) of the tiles sampled for one system."""
    out = [(1, 0, 0), (1, nm - TILE, nm - TILE), (3, 0, 0), (3, nts - TILE, nm - TILE),
           (4, 0, 0), (4, nts - TILE, nts - TILE)]
    out += extra
    for _ in range(6):
        r, c = int(rng.integers(0, nm - TILE + 1)), int(rng.integers(0, nm - TILE + 1))
        out.append((1, max(r, c), min(r, c)))
    for _ in range(3):
        out.append((3, int(rng.integers(0, nts - TILE + 1)), int(rng.integers(0, nm - TILE + 1))))
    out.append((4, int(rng.integers(0, nts - TILE + 1)), int(rng.integers(0, nts - TILE + 1))))
    return out


def elt_extra(t):
    """Tiles on each kind of WFS pair of the ELT system (WFS k's x slopes start at
    row 2*k*ns, its y slopes at 2*k*ns + ns; WFS 0-5 LGS, 6-7 NGS)."""
    ns = int(t.table("Nsubap")[0])
    w = lambda k, y=0, off=0: 2 * k * ns + y * ns + off
    return [
        (1, w(0, 0, 100), w(0, 0, 40)),          # LGS diagonal block, x-x
        (1, w(0, 1, 10) - 24, w(0, 0, ns - 30)),  # across the x/y boundary of one LGS
        (1, w(1, 0, 700), w(0, 0, 2000)),       # LGS x LGS (offset table pair)
        (1, w(5, 1, 1500), w(2, 0, 300)),       # LGS x LGS, y-x
        (1, w(6, 0, 1000), w(2, 0, 2500)),      # NGS x LGS (shared-point block)
        (1, w(7, 1, 2900), w(4, 1, 10)),        # NGS x LGS, y-y, at the grid edge
        (1, w(7, 0, 100), w(6, 1, 1234)),       # NGS x NGS
        (1, w(6, 1, 2960) - 40, w(6, 1, 2940) - 40),  # NGS diagonal block
        (3, 100, w(3, 0, 500)),                 # truth sensor x LGS (shared-point block)
        (3, ns + 50, w(1, 1, 2000)),            # truth sensor y x LGS y
        (3, 2000, w(6, 0, 400)),                # truth sensor x NGS
        (3, ns - 24, w(7, 1, 2950) - 40),       # across boundaries, last WFS
    ]


def sample_large(rng, v, k=600):
    idx = np.sort(rng.choice(v.size, size=min(k, v.size), replace=False))
    return idx, v[idx]


def golden(name, t, extra=(), seed=7):
    info = t.info
    nm, nts = info.nmeas, info.nmeasts
    rng = np.random.default_rng(seed)
    out = {k: t.table(k) for k in SMALL_TABLES}
    for k in LARGE_TABLES:
        v = t.table(k)
        out[f"{k}_sum"], out[f"{k}_fro"], out[f"{k}_n"] = np.array(v.sum()), np.array(
            np.linalg.norm(v)), np.array(v.size)
        out[f"{k}_idx"], out[f"{k}_val"] = sample_large(rng, v)
    spec = tiles_for(nm, nts, rng, list(extra))
    for typ, r0, c0 in spec:  # every tile inside its matrix
        nr, nc = {1: (nm, nm), 3: (nts, nm), 4: (nts, nts)}[typ]
        assert 0 <= r0 <= nr - TILE and 0 <= c0 <= nc - TILE, (name, typ, r0, c0)
    vals = np.zeros((len(spec), TILE, TILE))
    t.setTarget(0)
    for i, (typ, r0, c0) in enumerate(spec):
        d = np.zeros((TILE, TILE), order="F")
        t.matcov_tile(d, TILE, TILE, r0, c0, TILE, typ)  # xoffset = first row
        vals[i] = d
    out["tile_spec"] = np.array(spec, dtype=np.int64)
    out["tile_vals"] = vals
    out["info"] = np.array([info.nW, info.nLgs, info.nLayer, info.Nx, nm, nts])
    path = os.path.join(HERE, f"ref_{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), f"nmeas {nm} nmeasts {nts} tiles {len(spec)}")


def main():
    ref = os.environ.get("REF", "/root/reference")
    if not O.RefTomo.available():
        raise SystemExit("oracle/_ref/libmoao_ref.so missing: run `make -C oracle ref REF=...`")
    sets = {}
    for s in SETS:
        d = os.path.join(ref, "datafile", "check", s)
        sp, ap = parse_sys(os.path.join(d, "sys-params.txt")), parse_atm(
            os.path.join(d, "prof-1-atmos-night0.txt"))
        sets[s] = {"sys": P.as_dict(sp), "atm": P.as_dict(ap)}
        # golden outputs from the reference's own files
        t = O.RefTomo(os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt"))
        golden(s, t)
    with open(os.path.join(HERE, "check_sets.json"), "w") as f:
        json.dump(sets, f, indent=1)
    legacy = {}
    bdir = os.path.join(ref, "datafile", "benchmark")
    for name in sorted(os.listdir(bdir)):
        f = os.path.join(bdir, name, "sys-params.txt")
        if os.path.exists(f):
            legacy[name] = [[float(x) for x in v] for v in read_positional(f)]
    with open(os.path.join(HERE, "legacy_sets.json"), "w") as f:
        json.dump(legacy, f)
    # the seeded ELT-scale system of the benchmark
    sp, ap = P.config_elt()
    d = tempfile.mkdtemp(prefix="moao_elt_")
    P.write_system(d, sp, ap)
    t = O.RefTomo(os.path.join(d, "sys-params.txt"), os.path.join(d, "prof-1-atmos-night0.txt"))
    golden("elt", t, elt_extra(t))


if __name__ == "__main__":
    main()
