"""SEG-Y trace codec on the GPU against the host codec (which is pinned to the reference's
own readTraceData / writeTrace and IBM conversions by tests/test_host_cpu.py): the decoded
cube and the encoded records must be identical bit for bit."""
import dataclasses

import numpy as np
import pytest

from poststackmig3d_b200 import Migrator
from poststackmig3d_b200 import host as H
from poststackmig3d_b200 import synth as S

from helpers import geometry_for

pytestmark = pytest.mark.gpu


def _records(words_be, n_t, il, xl):
    """Records with IL/XL at 188/192 and the given big-endian sample words."""
    n = words_be.shape[0]
    rec = np.zeros((n, 240 + 4 * n_t), dtype=np.uint8)
    il = np.broadcast_to(np.asarray(il), (n,)).astype(">i4")
    xl = np.broadcast_to(np.asarray(xl), (n,)).astype(">i4")
    rec[:, 188:192] = il.view(np.uint8).reshape(n, 4)
    rec[:, 192:196] = xl.view(np.uint8).reshape(n, 4)
    rec[:, 7] = np.arange(n) % 251  # something to copy
    rec[:, 240:] = np.ascontiguousarray(words_be, dtype=">u4").view(np.uint8).reshape(n, -1)
    return rec


def _migrator(n_il, n_xl, n_t, pad_il=0, pad_xl=0):
    W = S.random_workload(50, n_il, n_xl, n_t, vel_kind="const", pad_il=pad_il, pad_xl=pad_xl)
    g = geometry_for(W)
    m = Migrator(0)
    m.set_geometry(g)
    return m, g


def _ibm_words(rng, n):
    w = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    # every exponent, single-bit fractions, zeros of both signs
    e = np.arange(n, dtype=np.uint32) % 128
    w[: n // 4] = (w[: n // 4] & 0x80FFFFFF) | (e[: n // 4] << 24)
    w[n // 4: n // 4 + 48] = (np.arange(48, dtype=np.uint32) % 24).astype(np.uint32)
    w[n // 4: n // 4 + 48] = (1 << w[n // 4: n // 4 + 48]) | (e[:48] << 24)
    w[-2:] = [0, 0x80000000]
    return w


def test_decode_ibm_matches_host():
    rng = np.random.default_rng(1)
    n_il, n_xl, n_t = 7, 9, 300
    m, g = _migrator(n_il, n_xl, n_t)
    with m:
        words = _ibm_words(rng, n_il * n_xl * n_t).reshape(n_il * n_xl, n_t)
        order = rng.permutation(n_il * n_xl)
        il = order // n_xl + 1
        xl = order % n_xl + 1
        rec = _records(words[order], n_t, il, xl)
        m.set_traces_segy(rec, 1, order)
        got = m.get_traces().reshape(n_il * n_xl, n_t)
        want = H.ibm_to_ieee(words.ravel()).reshape(n_il * n_xl, n_t)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_decode_ieee_positions_and_missing_traces():
    rng = np.random.default_rng(2)
    n_il, n_xl, n_t = 5, 6, 130
    m, g = _migrator(n_il, n_xl, n_t)
    with m:
        vals = rng.standard_normal((n_il * n_xl, n_t)).astype(np.float32)
        vals[0, :4] = [np.inf, -np.inf, np.nan, 1e-42]  # passed through bit for bit
        pos = np.arange(n_il * n_xl, dtype=np.int32)
        pos[3] = -1  # a skipped record
        keep = np.ones(n_il * n_xl, dtype=bool)
        keep[11] = False  # a cube trace with no record
        rec = _records(vals[keep].view(np.uint32), n_t, 1, 1)
        m.set_traces_segy(rec, 5, pos[keep])
        got = m.get_traces().reshape(n_il * n_xl, n_t)
        want = vals.copy()
        want[3] = 0.0
        want[11] = 0.0
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        # a repeated or out-of-range position is refused
        with pytest.raises(Exception):
            m.set_traces_segy(rec[:2], 5, [4, 4])
        with pytest.raises(Exception):
            m.set_traces_segy(rec[:1], 5, [n_il * n_xl])


@pytest.mark.parametrize("fmt", [1, 5])
def test_encode_matches_host(fmt):
    rng = np.random.default_rng(3 + fmt)
    n_il, n_xl, n_t = 4, 5, 257
    m, g = _migrator(n_il, n_xl, n_t, pad_il=1, pad_xl=2)
    with m:
        # input records, so that output traces can copy their headers
        vals = rng.standard_normal((n_il * n_xl, n_t)).astype(np.float32)
        il = np.repeat(np.arange(1, n_il + 1), n_xl)
        xl = np.tile(np.arange(1, n_xl + 1), n_il)
        rec = _records(vals.view(np.uint32), n_t, il, xl)
        m.set_traces_segy(rec, 5, np.arange(n_il * n_xl))
        img = (rng.standard_normal((g.n_oi, g.n_ox, n_t)) *
               10.0 ** rng.integers(-40, 38, (g.n_oi, g.n_ox, n_t))).astype(np.float32)
        img.ravel()[:8] = [0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -3e-39, 3.4e38]
        m.set_image(img)
        n_out = g.n_oi * g.n_ox
        source = np.full(n_out, -1, dtype=np.int32)
        source[5:5 + n_il * n_xl:2] = np.arange(0, n_il * n_xl, 2)[:len(source[5:5 + n_il * n_xl:2])]
        il_label = np.arange(100, 100 + g.n_oi, dtype=np.int32)
        xl_label = np.arange(-3, -3 + g.n_ox, dtype=np.int32)
        out = m.get_image_segy(fmt, source, il_label, xl_label)
    samples = out[:, 240:].copy().view(">u4").reshape(n_out, n_t).astype(np.uint32)
    flat = img.reshape(n_out, n_t)
    if fmt == 1:
        want = H.ieee_to_ibm(flat.ravel()).reshape(n_out, n_t)
    else:
        want = flat.view(np.uint32)
    assert np.array_equal(samples, want)
    for r in range(n_out):
        h = out[r, :240]
        if source[r] >= 0:
            assert np.array_equal(h, rec[source[r], :240]), r
        else:
            z = np.zeros(240, dtype=np.uint8)
            z[188:192] = np.array([il_label[r // g.n_ox]], ">i4").view(np.uint8)
            z[192:196] = np.array([xl_label[r % g.n_ox]], ">i4").view(np.uint8)
            assert np.array_equal(h, z), r
