"""The LBVH build's one device-side wait, the sort's decoupled look-back, is bounded:
after its poll limit a tile records CPT_STATUS_TIMEOUT and goes on; topology, refit
and the wide-tree build then return at once, and the build reports
CPT_ERR_DEVICE_TIMEOUT. The wait is made to run out by the build's test hook (tile 0
of the first sort pass never publishes its digit counts, a flag nothing else sets)
with a short poll limit: no fault, and the context stays usable. The next build on
the same objects is bit-exact against the oracle again."""
import numpy as np
import pytest

import cpt
from cpt.device import DeviceLbvh, to_device
from oracle import cpu
from test_gpu_build import assert_same_as

pytestmark = pytest.mark.gpu

STALL = cpt.BUILD_TEST_WITHHOLD | cpt.build_lookback_limit(10)  # 1,024 polls per tile


@pytest.mark.parametrize("bits", [30, 63])
def test_lookback_wait_runs_out_and_the_next_build_is_exact(cuda, bits):
    tris = cpt.scene_random(300_000, seed=11)[0]  # 74 sort tiles
    lb = DeviceLbvh(len(tris), bits)
    d = to_device(tris)
    with pytest.raises(cpt.CptError) as e:
        lb.build(d, check_root=True, flags=STALL)
    assert e.value.code == cpt.ERR_DEVICE_TIMEOUT
    assert lb.status_words()[0] & 2  # CPT_STATUS_TIMEOUT
    # without the check flag the call only enqueues; the status check reports it
    lb.build(d, flags=STALL)
    with pytest.raises(cpt.CptError) as e:
        lb.status()
    assert e.value.code == cpt.ERR_DEVICE_TIMEOUT
    # a wide tree over the failed build writes nothing and keeps the timeout
    lb.wide()
    with pytest.raises(cpt.CptError) as e:
        lb.status()
    assert e.value.code == cpt.ERR_DEVICE_TIMEOUT
    # the next build clears the status and is the oracle's, bit for bit
    lb.build(d, check_root=True)
    out = lb.download()
    assert_same_as(out, cpu.build(tris, bits))
    assert lb.status_words()[0] == 0


def test_short_poll_limit_alone_is_harmless(cuda):
    """A small limit without the hook: tiles publish as usual, so the build is exact
    (a wait that did run out would be reported, never silent)."""
    tris = cpt.scene_random(200_000, seed=12)[0]
    lb = DeviceLbvh(len(tris), 63)
    d = to_device(tris)
    try:
        lb.build(d, check_root=True, flags=cpt.build_lookback_limit(12))
    except cpt.CptError as e:
        assert e.code == cpt.ERR_DEVICE_TIMEOUT
        return
    assert_same_as(lb.download(), cpu.build(tris, 63))
    assert np.all(lb.status_words()[:1] == 0)
