"""Generates the golden fixtures in tests/golden/ from the reference.

Run in a container that has the reference tree and its compiled checker
(``make -C oracle ref ref-strict``):

    python tests/golden/make_golden.py [REF_SRC]

It writes two files:

- ``reference_unit_inputs.json``: the inputs of the reference's own unit
  tests for this path, read as text from its Catch2 test sources
  (src/TESTS/Mechanics/ForceField/{Volume,Branching,Boundary}/Test*.cpp and
  src/TESTS/Mechanics/Minimizer/TestCGMethod.cpp), plus the energies and forces
  the reference's compiled kernels return on them, in both the reference's
  build flags and strict IEEE rounding.
- ``synthetic_networks.npz``: two small seeded synthetic networks (complete
  force-field vectorizations) with the reference's energies and forces.

The GPU box does not have the reference; the tests read only these files.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from medyan_b200._abi import SystemView  # noqa: E402
from medyan_b200.network import make_workload  # noqa: E402
from oracle.oracle import Oracle, Reference  # noqa: E402

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def braced(text: str, start: int) -> str:
    """Contents of the first balanced {...} at or after start."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j]
    raise ValueError("unbalanced braces")


def numbers(s: str) -> list[float]:
    return [float(v) for v in re.findall(NUM, s)]


def after(text: str, anchor: str, start: int = 0) -> int:
    return text.index(anchor, start) + len(anchor)


def parse_excl(src: str) -> dict:
    t = strip_comments(open(src).read())
    out = {}
    # scaling test
    p = after(t, "TEST_CASE(\"Force field: Cylinder excl volume scaling\"")
    coord = numbers(braced(t, after(t, "const std::vector<floatingpoint> coord", p)))
    bs0 = numbers(braced(t, after(t, "beadSet0", p)))
    k0 = numbers(braced(t, after(t, "k0", p)))
    eq0 = numbers(braced(t, after(t, "eqLength0", p)))
    bs1 = numbers(braced(t, after(t, "beadSet1", p)))
    k1 = numbers(braced(t, after(t, " k1", p)))
    eq1 = numbers(braced(t, after(t, "eqLength1", p)))
    out["scaling"] = dict(coord=coord, beads0=bs0, k0=k0, eqlen0=eq0, beads1=bs1, k1=k1, eqlen1=eq1)
    # energy/force consistency inputs: testInputs.push_back({ "name", {beads}, {k}, {eq}, {coord} })
    p = after(t, "TEST_CASE(\"Force field: Cylinder excl volume\"")
    cases = {}
    pos = p
    while True:
        try:
            q = t.index("testInputs.push_back(", pos)
        except ValueError:
            break
        body = braced(t, q)
        name = re.search(r'"([^"]+)"', body).group(1)
        groups = []
        depth = 0
        cur = ""
        for ch in body[body.index(name) + len(name) + 1:]:
            if ch == "{":
                depth += 1
                if depth == 1:
                    cur = ""
                    continue
            elif ch == "}":
                depth -= 1
                if depth == 0:
                    groups.append(cur)
                    continue
            if depth >= 1:
                cur += ch
        if name != "almost-coplanar-unstable":
            cases[name] = dict(beads=numbers(groups[0]), k=numbers(groups[1]), eqlen=numbers(groups[2]),
                               coord=numbers(groups[3]))
        pos = q + 10
    out["consistency"] = cases
    # the disabled near-coplanar fixture from a real run (stress input)
    bs = numbers(braced(t, after(t, "beadSet20210901[]")))
    eq = numbers(braced(t, after(t, "eqLength20210901[]")))
    co = numbers(braced(t, after(t, "coord20210901[]")))
    out["stress_20210901"] = dict(beads=bs, eqlen=eq, coord=co, k=[100.0] * (len(bs) // 4))
    return out


def parse_branch(src: str, kname: str, per_case: int) -> dict:
    t = strip_comments(open(src).read())
    coords = []
    if per_case == 4:
        for m in re.finditer(r"coords\.insert\(coords\.end\(\),", t):
            coords.extend(numbers(braced(t, m.end())))
    else:
        for m in re.finditer(r"coords\.push_back\(V3", t):
            coords.extend(numbers(braced(t, m.end())))
    pos = [float(v) for v in re.findall(r"\bpos\.push_back\((" + NUM + r")\)", t)]
    k = [float(v) for v in re.findall(r"\b" + kname + r"\.push_back\((" + NUM + r")\)", t)]
    return dict(coord=coords, pos=pos, k=k)


def parse_boundary(src: str) -> dict:
    t = strip_comments(open(src).read())
    m = re.search(r"PlaneBoundaryElement element1\(\{([^}]*)\},\s*\{([^}]*)\},\s*(" + NUM + r"),\s*(" + NUM + r")\)", t)
    point, normal = numbers(m.group(1)), numbers(m.group(2))
    coords = numbers(braced(t, after(t, "std::vector< floatingpoint > coords")))
    kreps = numbers(braced(t, after(t, "kreps")))
    slens = numbers(braced(t, after(t, "slens")))
    beads = numbers(braced(t, after(t, "std::vector< int > beadSet")))
    nn = numbers(braced(t, after(t, "numNeighbors")))
    d = -sum(a * b for a, b in zip(normal, point))
    return dict(plane=normal + [d], element_k=float(m.group(3)), element_slen=float(m.group(4)), coord=coords,
                k=kreps, slen=slens, beads=beads, nneighbors=nn)


def parse_cg(src: str) -> dict:
    t = strip_comments(open(src).read())
    opt = numbers(braced(t, after(t, "optCoord")))
    w = numbers(braced(t, after(t, "weight")))
    n = int(re.search(r"constexpr int n = (\d+);", t).group(1))
    # inits: vector<floatingpoint>(800, n) -> 800 copies of n; only the first n are degrees of freedom
    m = re.search(r"vector<floatingpoint>\((\d+), n\)", t)
    init0 = [float(n)] * n if m else None
    init2 = numbers(braced(t, t.index("vector<floatingpoint>{", t.index("inits"))))
    params = dict(gradTol=float(re.search(r"cgParams\.gradTol = (" + NUM + ")", t).group(1)),
                  maxDist=float(re.search(r"cgParams\.maxDist = (" + NUM + ")", t).group(1)),
                  lambdaMax=float(re.search(r"cgParams\.lambdaMax = (" + NUM + ")", t).group(1)))
    return dict(n=n, opt=opt, weight=w, inits=[init0, list(opt), init2], params=params)


def ref_eval(ref: Reference, sv: SystemView, x):
    e, per = ref.energy(sv, x)
    f = ref.forces(sv, x)
    return dict(energy=e, per_ff=per.tolist(), force=f.tolist())


def main(ref_src: str) -> None:
    ff = os.path.join(ref_src, "TESTS", "Mechanics", "ForceField")
    data = {
        "excl": parse_excl(os.path.join(ff, "Volume", "TestCylinderExclVolume.cpp")),
        "dihedral": parse_branch(os.path.join(ff, "Branching", "TestBranchingDihedralCosine.cpp"), "kdih", 4),
        "position": parse_branch(os.path.join(ff, "Branching", "TestBranchingPositionCosine.cpp"), "kpos", 3),
        "boundary": parse_boundary(os.path.join(ff, "Boundary", "TestBoundaryBeadRepulsion.cpp")),
        "cg_harmonic": parse_cg(os.path.join(ref_src, "TESTS", "Mechanics", "Minimizer", "TestCGMethod.cpp")),
    }
    refs = {"reference": Reference(strict=False), "strict": Reference(strict=True)}
    results = {}
    for tag, ref in refs.items():
        r = {}
        ex = data["excl"]
        sc = ex["scaling"]
        n = len(sc["coord"]) // 3
        sv0 = SystemView(n, excl_beads=sc["beads0"], excl_k=sc["k0"], excl_eqlen=sc["eqlen0"])
        sv1 = SystemView(n, excl_beads=sc["beads1"], excl_k=sc["k1"], excl_eqlen=sc["eqlen1"])
        r["excl_scaling"] = dict(energy0=ref.energy(sv0, sc["coord"])[0], energy1=ref.energy(sv1, sc["coord"])[0])
        for name, c in ex["consistency"].items():
            sv = SystemView(len(c["coord"]) // 3, excl_beads=c["beads"], excl_k=c["k"], excl_eqlen=c["eqlen"])
            r["excl_" + name] = ref_eval(ref, sv, c["coord"])
        st = ex["stress_20210901"]
        sv = SystemView(len(st["coord"]) // 3, excl_beads=st["beads"], excl_k=st["k"], excl_eqlen=st["eqlen"])
        r["excl_stress"] = ref_eval(ref, sv, st["coord"])
        dh = data["dihedral"]
        nb = len(dh["pos"])
        sv = SystemView(len(dh["coord"]) // 3, branch_beads=[3 * i for i in range(4 * nb)], branch_pos=dh["pos"],
                        branch_dihedral_k=dh["k"], branch_ff_mask=4)
        r["dihedral"] = ref_eval(ref, sv, dh["coord"])
        ps = data["position"]
        nb = len(ps["pos"])
        beads = []
        for i in range(nb):
            beads += [9 * i, 9 * i + 3, 9 * i + 6, 9 * i + 6]
        sv = SystemView(len(ps["coord"]) // 3, branch_beads=beads, branch_pos=ps["pos"], branch_position_k=ps["k"],
                        branch_ff_mask=8)
        r["position"] = ref_eval(ref, sv, ps["coord"])
        bd = data["boundary"]
        sv = SystemView(len(bd["coord"]) // 3, boundary_beads=bd["beads"], boundary_k=bd["k"],
                        boundary_slen=bd["slen"], plane_eq=bd["plane"], plane_nneighbors=bd["nneighbors"])
        r["boundary"] = ref_eval(ref, sv, bd["coord"])
        results[tag] = r
    data["results"] = results
    with open(os.path.join(HERE, "reference_unit_inputs.json"), "w") as fh:
        json.dump(data, fh, indent=1)

    # seeded synthetic networks with complete vectorizations
    orc = Oracle()
    arrays = {}
    nets = {
        "cfg0": make_workload(0),
        "branched": make_workload(1, n_fil=80, cyl_per_fil=8, box=1600.0, n_linker=60, n_motor=12, n_branch=16,
                                  br_position_k=20.0, seed=11),
    }
    for tag, net in nets.items():
        st, extra = orc.complete(net)
        assert st == 0
        if tag == "branched":
            # one branch at the parent's plus end exercises the virtual plus end
            net.ff["branch_pos"] = net.ff["branch_pos"].copy()
            net.ff["branch_pos"][0] = 1.0
        sv = net.system_view(**extra)
        x = net.flat_coords()
        for k, v in sv.arrays.items():
            arrays[f"{tag}/{k}"] = v
        arrays[f"{tag}/n_beads"] = np.array([net.n_beads])
        arrays[f"{tag}/branch_ff_mask"] = np.array([sv.branch_ff_mask])
        arrays[f"{tag}/coord"] = x
        for rtag, ref in refs.items():
            e, per = ref.energy(sv, x)
            arrays[f"{tag}/{rtag}/energy"] = np.array([e])
            arrays[f"{tag}/{rtag}/per_ff"] = per
            arrays[f"{tag}/{rtag}/force"] = ref.forces(sv, x)
    np.savez_compressed(os.path.join(HERE, "synthetic_networks.npz"), **arrays)
    print("wrote", os.path.join(HERE, "reference_unit_inputs.json"), "and synthetic_networks.npz")


if __name__ == "__main__":
    default = os.environ.get("MEDYAN_REF_SRC",
                             os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference", "src"))
    main(sys.argv[1] if len(sys.argv) > 1 else default)
