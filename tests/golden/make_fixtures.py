"""Turn the reference's JLD2 golden files into the numpy fixtures that the tests read.

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

REFERENCE_ROOT is the root of the juliaTDGL checkout (it holds ``gtdgl/test/golden``).  Writes, next to
this script:

* ``<case>.npz`` for the release-1.2 regression states used by ``gtdgl/test/test_regression12.jl``
  (``k2_R13_explicit``, ``k2_R4_prod``, ``k25_R4_prod``): the step parameters (``par``, as JSON), the
  state before (``ini_*``) and after (``fin_*``) 40 steps, and the masks of the case;
* ``masks_wedge.npz``: the WEDGE / SIM condensation masks of ``gtdgl/test/golden/masks.jld2``
  (``gtdgl/test/test_geometry.jl``), with the mesh and geometry keywords of each case;
* ``masks_catalogue.npz``: every catalogue case of the same golden file (all modes and their _REF mirrors on two
  meshes, the z modes, the shifts, the prism angle, the fgrad direction), with the mesh and keywords of each;
* ``masks_custom.npz``: the shape-file cases of the same golden file (GEOM_MODE CUSTOM and CUSTOM_REF, written by
  release 1.2), each mask with its mesh and keywords, and the text of every shape file they read
  (``gtdgl/shapes/<geom_file>``, the files the reference's test rasterises against these masks).

Only this script reads the reference; the tests read the fixtures.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from juliatdgl_b200 import jld2 as jld2_reader  # noqa: E402

REG_CASES = ("k2_R13_explicit", "k2_R4_prod", "k25_R4_prod", "k2_R4_drag", "k2_R4_heat")
MASK_CASES = ("SIM_40x24x6", "SIM_30x20x8", "WEDGE_40x24x6", "WEDGE_30x20x8", "WEDGE_zhalf", "WEDGE_zburied")


def main(ref_root):
    gold = os.path.join(ref_root, "gtdgl", "test", "golden")
    for name in REG_CASES:
        d = jld2_reader.load(os.path.join(gold, f"{name}.jld2"))
        out = {"par": np.array(json.dumps(d["par"]))}
        for tag in ("ini", "fin"):
            for k, v in d[tag].items():
                out[f"{tag}_{k}"] = np.asarray(v)
        for k in ("fmask", "taux", "tauy", "tauz", "taupsi"):
            out[k] = np.asarray(d[k])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)
    casos = jld2_reader.load(os.path.join(gold, "masks.jld2"))["casos"]
    out = {}
    meta = {}
    for name in MASK_CASES:
        c = casos[name]
        out[name] = np.asarray(c["fmask"])
        meta[name] = {"malla": c["malla"], "geo": c["geo"]}
    b = casos["_box_40x24x6"]
    for k in ("taux", "tauy", "tauz", "taupsi"):
        out[f"_box_{k}"] = np.asarray(b[k])
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "masks_wedge.npz"), **out)
    print("wrote masks_wedge")
    out, meta = {}, {}
    for name in sorted(k for k in casos if not k.startswith("CUSTOM") and not k.startswith("_")):
        c = casos[name]
        out[name] = np.asarray(c["fmask"])
        meta[name] = {"malla": c["malla"], "geo": c["geo"]}
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "masks_catalogue.npz"), **out)
    print("wrote masks_catalogue", len(meta))
    out, meta, texts = {}, {}, {}
    for name in sorted(k for k in casos if k.startswith("CUSTOM")):
        c = casos[name]
        out[name] = np.asarray(c["fmask"])
        meta[name] = {"malla": c["malla"], "geo": c["geo"]}
        f = c["geo"]["geom_file"]
        if f not in texts:
            with open(os.path.join(ref_root, "gtdgl", "shapes", f)) as fh:
                texts[f] = fh.read()
    out["meta"] = np.array(json.dumps(meta))
    out["shape_files"] = np.array(json.dumps(texts))
    np.savez_compressed(os.path.join(HERE, "masks_custom.npz"), **out)
    print("wrote masks_custom", len(meta))


def ladder_fixture(ref_root):
    """``ladder_k25.npz``: the two-polarity golden ladder of gtdgl/test/golden/ladder_k25.jld2 (made by
    gtdgl/test/golden/make_ladder.jl, checked by gtdgl/test/test_protocol.jl:4-29): per polarity the currents,
    verdicts, cycles, voltages, slopes, slip counts, magnetisation, vortex counts, residuals and the final Ψ of both
    bands; the step, substeps, mass ratio and fixed-point tolerance; the brackets."""
    gold = os.path.join(ref_root, "gtdgl", "test", "golden")
    d = jld2_reader.load(os.path.join(gold, "ladder_k25.jld2"))
    out = {}
    for pol in ("pos", "neg"):
        for k, v in d[pol].items():
            out[f"{pol}_{k}"] = np.array(v) if k != "conv" else np.array(str(v))
    for k in ("eps_c", "dt", "n_pi", "mr", "lo_pos", "hi_pos", "lo_neg", "hi_neg"):
        out[k] = np.array(d[k])
    np.savez_compressed(os.path.join(HERE, "ladder_k25.npz"), **out)
    print("wrote ladder_k25")


def jld2_fixture(ref_root):
    """``k2_R4_heat.jld2``: one of the reference's own JLD2 files, kept as the reference wrote it, so that the
    package's JLD2 reader (``juliatdgl_b200.jld2``, used by ``checkpoint.load``) is tested on a file gtdgl wrote.
    Its ``ini`` group is a state in the reference's key names (G1…, thetax…, phix…, hx…, Temp)."""
    import shutil
    shutil.copy(os.path.join(ref_root, "gtdgl", "test", "golden", "k2_R4_heat.jld2"), os.path.join(HERE, "k2_R4_heat.jld2"))
    print("copied k2_R4_heat.jld2")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TDGL_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_fixtures.py REFERENCE_ROOT (the juliaTDGL checkout; or set TDGL_REFERENCE_ROOT)")
    main(root)
    ladder_fixture(root)
    jld2_fixture(root)
