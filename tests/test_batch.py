"""Batched lattices (kofm_batch_*): several channels advanced by one CUDA
graph per two steps give exactly the results of stepping them one by one, and
the seeded sweep of uneven channels is reproducible."""
import numpy as np
import pytest

from komegafoulingmodel_b200 import Lattice, _abi, desc_default
from komegafoulingmodel_b200 import geometry as G
from komegafoulingmodel_b200.batch import Batch, sweep_channels
from tests.test_komega_gpu import channel_case


def test_sweep_is_seeded_and_follows_its_rules():
    a = sweep_channels(6, seed=3)
    b = sweep_channels(6, seed=3)
    for wa, wb in zip(a, b):
        assert wa.name == wb.name and np.array_equal(wa.f, wb.f)
        nx, ny = wa.channel.nx, wa.channel.ny
        assert nx in (512, 1024, 2048, 4096) and ny in (64, 128, 256)
        re = float(wa.name.split("_re")[1])
        assert 500 <= re <= 30000 and wa.komega == (re >= 2000)


def _cases():
    out = []
    ch = G.straight_channel(256, 40)
    out.append(("laminar", ch, G.equilibrium_state(ch, ux=0.01), None, None, None, 1.25, 1e-6, 0.1))
    for nx, ny, amp in ((128, 34, 0.0), (256, 66, 8.0)):
        c, f, k, o, nut, rate, g, nu = channel_case(nx=nx, ny=ny)
        if amp > 0:
            c = G.wavy_channel(nx, ny, amp, 128)
            f = G.equilibrium_state(c, ux=0.02)
            k, o, nut = G.komega_fields(c, 1.5 * (0.05 * 0.05) ** 2, 0.003)
        out.append(("komega", c, f, k, o, nut, rate, g, nu))
    return out


def _open(case, storage=_abi.STORE_FP32, form=2):
    kind, ch, f, k, o, nut, rate, g, nu = case
    d = desc_default()
    d.storage = storage
    d.komega_classic = form
    d.nx, d.nx_full, d.ny = ch.nx, ch.nx_full, ch.ny
    d.tau, d.fterm, d.mu = rate, g, nu
    d.use_komega = 1 if kind == "komega" else 0
    L = Lattice(d)
    ko = kind == "komega"
    L.set_geometry(ch.ntype, ch.wallD if ko else None, ch.dX if ko else None,
                   ch.ibb_idx if len(ch.ibb_idx) else None, ch.ibb_q if len(ch.ibb_q) else None)
    L.set_state(f, k, o, nut, np.zeros(3 * ch.n) if ko else None)
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [_abi.STORE_FP32, _abi.STORE_FP16_NEQ])
def test_batch_matches_one_by_one(kofm_lib, storage):
    """A graph replays the one-launch form of the solve (komega_classic = 2):
    bit-identical to stepping contexts of that form one by one."""
    cases = _cases()
    solo = [_open(c, storage) for c in cases]
    both = [_open(c, storage) for c in cases]
    try:
        for L in solo + both:
            L.step(1)
        with pytest.raises(_abi.KofmError):
            Batch([both[0], both[0]])          # the same context twice
        with Batch(both) as B:
            B.step(4)
            with pytest.raises(_abi.KofmError):
                B.step(3)                      # odd step counts are rejected
        for L in solo:
            L.step(4)
        for a, b in zip(solo, both):
            sa, sb = a.get_state(), b.get_state()
            for x, y in zip(sa, sb):
                if x is not None:
                    assert np.array_equal(x, y)
            assert a.stats().steps == b.stats().steps == 5
    finally:
        for L in solo + both:
            L.close()


@pytest.mark.gpu
def test_batch_needs_stepped_contexts(kofm_lib):
    L = _open(_cases()[0])
    try:
        with pytest.raises(_abi.KofmError):
            Batch([L])                          # populations still in the set_state form
    finally:
        L.close()


@pytest.mark.gpu
def test_batch_of_phase_form_contexts_agrees_to_rounding(kofm_lib):
    """Contexts of the default form (phase launches, stepped on their own)
    batched: the graph runs the same solve in one launch, whose partial sums
    group differently; fields agree to rounding (rel-L2 1e-6)."""
    cases = _cases()
    solo = [_open(c, form=0) for c in cases]
    both = [_open(c, form=0) for c in cases]
    try:
        for L in solo + both:
            L.step(1)
        with Batch(both) as B:
            B.step(4)
        for L in solo:
            L.step(4)
        for a, b in zip(solo, both):
            for x, y in zip(a.get_state(), b.get_state()):
                if x is not None:
                    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
                    assert np.linalg.norm(x - y) <= 1e-6 * max(np.linalg.norm(x), 1e-30)
    finally:
        for L in solo + both:
            L.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tile_rows", [1, 3, -1])
def test_tile_shapes_of_the_multi_lattice_collide_give_identical_steps(kofm_lib, tile_rows):
    """The persistent multi-lattice collide walks tiles of tile_rows block
    rows (-1: one collide launch per lattice): every tile shape computes each
    node as the one-lattice collide does, so the batch stays bit-identical to
    stepping the contexts one by one."""
    cases = _cases()
    solo = [_open(c) for c in cases]
    both = [_open(c) for c in cases]
    try:
        for L in solo + both:
            L.step(1)
        with Batch(both, tile_rows) as B:
            B.step(4)
        for L in solo:
            L.step(4)
        for a, b in zip(solo, both):
            for x, y in zip(a.get_state(), b.get_state()):
                if x is not None:
                    assert np.array_equal(x, y)
            assert a.get_macro()[0].tobytes() == b.get_macro()[0].tobytes()
    finally:
        for L in solo + both:
            L.close()
