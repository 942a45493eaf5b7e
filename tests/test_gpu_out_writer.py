"""The .out writer on the device (grb_format_out + grb_drain_out).

Against a restatement of the reference's writer (graph::output_nets,
output.hpp:79-112, and RouteWriter::segment, output_writer.hpp:29-43): after
an L-shape stage on a seeded design, records with names, pins on several
layers (a via is written for layer-0 pins only), extra route pairs, several
subnets each and empty records give byte-identical text; a record that names
an unknown subnet is refused.  The drop-in test covers the writer inside the
reference's own program flow.
"""
import numpy as np
import pytest

from helpers import net_routes

pytestmark = pytest.mark.gpu


def reference_text(X, Y, names, pins, extra, subnets, routes, route_off):
    XY = X * Y

    def seg(a, b):
        a, b = int(a), int(b)
        if a > b:
            a, b = b, a
        return f"{a // Y % X} {a % Y} {a // XY} {b // Y % X} {b % Y} {b // XY}\n"
    out = []
    for name, ps, ex, subs in zip(names, pins, extra, subnets):
        out.append(name + "\n(\n")
        out.extend(seg(p, p + XY) for p in ps if p < XY)
        out.extend(seg(ex[i], ex[i + 1]) for i in range(0, len(ex) - 1, 2))
        for s in subs:
            r = net_routes(routes, route_off, s)
            out.extend(seg(r[j] + XY, r[j + 1] + XY) for j in range(1, int(r[0]) - 1, 2))
        out.append(")\n")
    return "".join(out).encode()


def test_device_writer_equals_reference_writer():
    from grotor_b200 import GrbError, Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["small_64x64x5"].scaled(3000))
    g, n = d.grid, d.nets
    r = Router(g)
    r.upload_nets(n)
    r.generate_batches_rsmt(d.order, 1000000, 1, "persistent")
    r.lshape_route("persistent")
    routes = r.read_routes()
    rng = np.random.default_rng(5)
    XY = g.X * g.Y
    names, pins, extra, subnets = [], [], [], []
    ids = rng.permutation(n.n)
    k = 0
    while k < n.n:
        m = int(rng.integers(0, 4))  # 0: a record without subnets
        subnets.append(ids[k:k + m])
        k += m
        names.append(f"net{len(names)}_" + "x" * int(rng.integers(0, 40)))
        pins.append(rng.integers(0, 3 * XY, int(rng.integers(0, 6))))
        extra.append(rng.integers(0, g.L * XY, 2 * int(rng.integers(0, 3))))
    text = r.write_out(names, pins, extra, subnets)
    want = reference_text(g.X, g.Y, names, pins, extra, subnets, routes, n.route_off)
    assert text == want
    assert r.write_out([], [], [], []) == b""
    with pytest.raises(GrbError):
        r.write_out(["bad"], [[]], [[]], [[n.n + 5]])
    assert r.write_out(names[:3], pins[:3], extra[:3], subnets[:3]) == reference_text(
        g.X, g.Y, names[:3], pins[:3], extra[:3], subnets[:3], routes, n.route_off)
    r.close()


def test_used_word_transfers():
    """grb_read_routes_used moves each net's count word and the words below it
    (and nothing else) to the host; grb_write_routes_used moves them back; a
    net whose count word is 0 still has that word moved."""
    from grotor_b200 import Router
    from grotor_b200.synth import WORKLOADS, Design
    d = Design(WORKLOADS["medium_320x320x10"].scaled(6000, seed=11))
    r = Router(d.grid)
    r.upload_nets(d.nets)
    r.generate_batches_rsmt(d.order, 1000000)
    r.lshape_route("persistent")
    full = r.read_routes()
    off = np.asarray(d.nets.route_off, np.int64)
    used = np.zeros(full.size, bool)
    for i in range(len(off) - 1):
        if off[i + 1] > off[i]:
            used[off[i]:off[i] + max(1, min(int(full[off[i]]), int(off[i + 1] - off[i])))] = True
    assert not used.all()
    got = r.read_routes_used(np.full(full.size, -7, np.int32))
    np.testing.assert_array_equal(got[used], full[used])
    assert (got[~used] == -7).all()
    # Back to the device over a reset (routes zeroed): the words in use return,
    # the others stay zero.
    r.reset()
    sent = np.where(used, full, 12345).astype(np.int32)
    r.write_routes_used(sent)
    back = r.read_routes()
    np.testing.assert_array_equal(back[used], full[used])
    assert (back[~used] == 0).all()
    r.close()
