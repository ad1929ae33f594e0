"""Failure detection of the persistent sweep's bounded dependency wait.

A work item waits, after its sweep and before its surface writes, for its
tile's previous sector.  The test holds one tile's completion counter (the
flag nothing sets), gives the wait a short limit, and checks that the run
ends with TVS_ERR_TIMEOUT within milliseconds instead of hanging, and that the
same context afterwards computes the oracle's results again.  Nothing here
faults or traps the GPU: the wait gives up by itself and the host reads the
status word."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("precision", ["exact32", "mixed64"])
def test_wait_that_cannot_be_satisfied_times_out(tvs, oracle, synth, precision):
    w, s, los = 301, 30.0, 3000
    z = synth.config_dem("plain_cpu")
    g = oracle.geometry(w, s, los)
    if precision == "exact32":
        want, want_total, _ = oracle.run(g, z, 1.65)
    else:
        want = oracle.run_f64(g, z, 1.65)[0].astype(np.float32)
        want_total = None
    with tvs.Engine(z, w, s, los, observer_height=1.65, precision=precision) as eng:
        eng.set_queue_wait(spin_limit=1000, held_tile=3)
        eng.device_reset()
        t0 = time.perf_counter()
        eng.device_run_sectors(0, 180)
        with pytest.raises(tvs.TvsError) as e:
            eng.device_finish()
        elapsed = time.perf_counter() - t0
        assert e.value.code == tvs.ERR_TIMEOUT
        assert elapsed < 2.0, elapsed   # the default limit alone would take ~2 s
        # the surfaces of the held tile never advanced past sector 0: incomplete
        got, _ = eng.read_surfaces()
        assert not np.array_equal(bits(got), bits(want))
        # back to the default limit and no held tile: exact results again
        eng.set_queue_wait()
        eng.device_reset()
        eng.device_run_sectors(0, 180)
        eng.device_finish()
        got, total = eng.read_surfaces()
    assert np.array_equal(bits(got), bits(want))
    if want_total is not None:
        assert np.array_equal(bits(total), bits(want_total))
