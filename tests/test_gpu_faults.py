"""The bounded-wait error path of the tensor-core search (GPU).

Every mbarrier wait in the tensor-core kernels is bounded: on expiry the kernel sets an
error word, stops taking tiles, frees its tensor memory and returns, and the call reports
EPIK2_E_TIMEOUT.  Here a test hook makes one producing warp of the first CTA leave out its
first "stage stored" arrival (on single CTAs, before any matrix product is issued), with the
wait limit shortened to ~10 ms of SM clock: the search must return EPIK2_E_TIMEOUT, and the
same context must then search correctly -- its tensor memory was released, or the next
launch could not allocate it.  No GPU fault is involved: the wait simply runs out.
"""
import pytest

import epik2
import oracle as O
from conftest import f32_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine,stage_words", [(epik2.ENGINE_TC, 8), (epik2.ENGINE_TC_FP4, 8)],
                         ids=["int8", "fp4"])
def test_expired_wait_returns_timeout_and_context_recovers(engine, stage_words):
    g, p = O.gen_hwe(121, 2000, 200, 1000, planted=[(5, 33, 171)], effects=[0.8])
    ref = O.scan(g, p)
    with epik2.Context(0, engine=engine, stage_words=stage_words) as ctx:
        did = ctx.load(g, p)
        before = ctx.scan(did)
        ctx.set_wait_limit(20_000_000)  # ~10 ms at 2 GHz
        ctx.test_withhold_arrival()
        with pytest.raises(epik2.Epik2Error) as e:
            ctx.scan(did)
        assert e.value.status == epik2.E_TIMEOUT
        after = ctx.scan(did)           # the hook is one-shot; same short limit still applies
        ctx.set_wait_limit(0)
        again = ctx.scan(did)
        ctx.unload(did)
    for b in (before, after, again):
        assert b.ijk == ref["ijk"] and f32_bits(b.score) == f32_bits(ref["score"])
