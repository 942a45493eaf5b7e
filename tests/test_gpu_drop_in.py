"""The drop-in: the reference router's own program flow with its routing hot
path on grotor_b200 (integration/grotor_grb, built against the reference's
headers by integration/Makefile) against the stock reference program
(oracle/_ref/grotor, its own src/main.cu), CAP/NET in, .out out.

Same input, same output: the same nets in the same order; every net's
segments identical -- byte for byte for nets routed only by stage one (the
L-shape stage), as a set for nets rerouted by stage two (the reference's FLT
stage appends segments with atomics, so their order is not defined) -- and
the reference evaluator's scores (wirelength, via, overflow and total cost,
open and incomplete nets) identical.  Runs on a congested design (many FLT
nets) and on the seeded 320x320x10 design with 120,000 nets.  The GGR
pipeline's drop-in (integration/grotor_grb_ggr) against the reference's own
GGR build: the whole .out byte for byte.
"""
import os
import subprocess
from dataclasses import replace

import pytest

from helpers import ROOT

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
STOCK = os.path.join(REF_DIR, "grotor")
DRIVER = os.path.join(ROOT, "integration", "_build", "grotor_grb")
STOCK_GGR = os.path.join(REF_DIR, "grotor_ggr")
DRIVER_GGR = os.path.join(ROOT, "integration", "_build", "grotor_grb_ggr")
STOCK_CUGR2 = os.path.join(REF_DIR, "grotor_cugr2")
DRIVER_CUGR2 = os.path.join(ROOT, "integration", "_build", "grotor_grb_cugr2")
EVALUATOR = os.path.join(REF_DIR, "evaluator")

DESIGNS = {
    "congested_48x48x10_1500": ("small_64x64x5", dict(n_nets=1500, cap_layers=10, seed=13, X=48, Y=48, cap_lo=1,
                                                     cap_hi=4)),
    "medium_320x320x10": ("medium_320x320x10", {}),
}
GGR_DESIGNS = {
    "ggr_48x48x10_1500": ("small_64x64x5", dict(n_nets=1500, cap_layers=10, seed=13, X=48, Y=48)),
    "ggr_160x160x10_20k": ("medium_320x320x10", dict(n_nets=20000, X=160, Y=160, big_lo=80, big_hi=160, seed=21)),
}


def parse_out(path):
    """[(net name, [segment lines])] in file order."""
    nets, name, segs = [], None, None
    for line in open(path):
        line = line.rstrip("\n")
        if name is None:
            name = line
        elif line == "(":
            segs = []
        elif line == ")":
            nets.append((name, segs))
            name, segs = None, None
        else:
            segs.append(line)
    assert name is None, "truncated .out"
    return nets


def scores(cap, net, out):
    res = subprocess.run([EVALUATOR, cap, net, out], capture_output=True, text=True)
    keep = ("overflow cost", "open nets", "incompleted nets", "wirelength cost", "via cost", "total cost", "FOR_STAT")
    lines = [ln.strip() for ln in (res.stdout + res.stderr).splitlines()
             if any(k in ln for k in keep) and "time" not in ln.lower()]
    assert len(lines) >= 6, res.stdout + res.stderr
    return lines


@pytest.mark.parametrize("name", list(DESIGNS))
def test_drop_in_matches_stock_reference(name, tmp_path):
    if not (os.path.exists(STOCK) and os.path.exists(DRIVER)):
        pytest.skip("stock reference or drop-in driver not built (oracle/ref.mk, integration/Makefile)")
    from grotor_b200.synth import WORKLOADS, Design
    wl, over = DESIGNS[name]
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    Design(replace(WORKLOADS[wl], **over)).write(cap, net)
    ref_out, mine = str(tmp_path / "ref.out"), str(tmp_path / "mine.out")
    r = subprocess.run([STOCK, "-cap", cap, "-net", net, "-out", ref_out, "--lut-dir", REF_DIR],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    m = subprocess.run([DRIVER, "-cap", cap, "-net", net, "-out", mine, "--lut-dir", REF_DIR],
                       capture_output=True, text=True, timeout=900)
    assert m.returncode == 0, m.stderr[-3000:]
    a, b = parse_out(ref_out), parse_out(mine)
    assert [n for n, _ in a] == [n for n, _ in b], "net order differs"
    reordered = 0
    for (n, sa), (_, sb) in zip(a, b):
        assert sorted(sa) == sorted(sb), f"net {n}: segments differ"
        reordered += sa != sb
    if "stage=detour" not in r.stdout:  # no stage-two nets: the whole file is identical
        assert open(ref_out, "rb").read() == open(mine, "rb").read()
    assert scores(cap, net, ref_out) == scores(cap, net, mine)
    print(f"{name}: {len(a)} nets, {reordered} with stage-two segments in another order")


@pytest.mark.parametrize("name", list(GGR_DESIGNS))
def test_ggr_drop_in_matches_stock_reference(name, tmp_path):
    """The GGR pipeline (the reference's grotor_ggr build, pipeline_ggr.hpp):
    first-fit groups, bounding-box batches and the Z-shape stage on
    grotor_b200, the reference's post-processing, the device writer; the .out
    must be byte-identical to the stock GGR program's, with identical scores."""
    if not (os.path.exists(STOCK_GGR) and os.path.exists(DRIVER_GGR)):
        pytest.skip("stock GGR reference or GGR drop-in driver not built (oracle/ref.mk, integration/Makefile)")
    from grotor_b200.synth import WORKLOADS, Design
    wl, over = GGR_DESIGNS[name]
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    Design(replace(WORKLOADS[wl], **over)).write(cap, net)
    ref_out, mine = str(tmp_path / "ref.out"), str(tmp_path / "mine.out")
    r = subprocess.run([STOCK_GGR, "-cap", cap, "-net", net, "-out", ref_out, "--lut-dir", REF_DIR, "--report-score",
                        "0"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    for ex in ("persistent", "plain"):
        m = subprocess.run([DRIVER_GGR, "-cap", cap, "-net", net, "-out", mine, "--lut-dir", REF_DIR, "--executor", ex],
                           capture_output=True, text=True, timeout=900)
        assert m.returncode == 0, m.stderr[-3000:]
        a, b = open(ref_out, "rb").read(), open(mine, "rb").read()
        assert a == b, f"{ex}: .out differs ({len(a)} vs {len(b)} bytes)"
    assert scores(cap, net, ref_out) == scores(cap, net, mine)


def stage_lines(text, tags):
    return [ln.strip() for ln in text.splitlines() if ln.split(" ")[0] in tags and "executor=" not in ln]


CUGR2_DESIGNS = dict(DESIGNS)
# a design whose maze stage the score gate accepts (the others reject theirs)
CUGR2_DESIGNS["maze_accepted_64x64x10_3000"] = ("small_64x64x5", dict(n_nets=3000, cap_layers=10, seed=2, X=64, Y=64,
                                                                      cap_lo=5, cap_hi=9))


@pytest.mark.parametrize("name", list(CUGR2_DESIGNS))
def test_cugr2_drop_in_matches_stock_reference(name, tmp_path):
    """The CUGR2 pipeline (the reference's grotor_cugr2 build,
    pipeline_cugr2.hpp): L-shape, rip-up, FLT detour and the maze stage with
    its checkpoint and score gate on grotor_b200 around the reference's host
    maze topology.  Same nets in the same order, every net's segments as a
    set, identical scores; the maze stage's sizes and its score gate (both
    scores, printed to 12 digits) as the stock program reports them."""
    if not (os.path.exists(STOCK_CUGR2) and os.path.exists(DRIVER_CUGR2)):
        pytest.skip("stock CUGR2 reference or CUGR2 drop-in driver not built (oracle/ref.mk, integration/Makefile)")
    from grotor_b200.synth import WORKLOADS, Design
    wl, over = CUGR2_DESIGNS[name]
    cap, net = str(tmp_path / "d.cap"), str(tmp_path / "d.net")
    Design(replace(WORKLOADS[wl], **over)).write(cap, net)
    ref_out, mine = str(tmp_path / "ref.out"), str(tmp_path / "mine.out")
    r = subprocess.run([STOCK_CUGR2, "-cap", cap, "-net", net, "-out", ref_out, "--lut-dir", REF_DIR, "--report-score",
                        "0"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    tags = ("ROUTING_STAGE_BEGIN", "MAZE_QUALITY_GATE", "ROUTING_REMAINING_OVERFLOW", "REROUTE_STORAGE")
    for ex in ("persistent", "plain"):
        m = subprocess.run([DRIVER_CUGR2, "-cap", cap, "-net", net, "-out", mine, "--lut-dir", REF_DIR, "--executor",
                            ex], capture_output=True, text=True, timeout=900)
        assert m.returncode == 0, m.stderr[-3000:]
        assert stage_lines(r.stdout, tags) == stage_lines(m.stdout, tags)
        a, b = parse_out(ref_out), parse_out(mine)
        assert [n for n, _ in a] == [n for n, _ in b], "net order differs"
        for (n, sa), (_, sb) in zip(a, b):
            assert sorted(sa) == sorted(sb), f"{ex}: net {n}: segments differ"
        assert scores(cap, net, ref_out) == scores(cap, net, mine)
    print(name, stage_lines(r.stdout, tags))
