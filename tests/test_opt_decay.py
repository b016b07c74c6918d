"""Learning-rate schedules (nnp_decay_step, host only) against the reference's
own opt::Decay::step (opt/decay.cpp:58-82, compiled in oracle/_ref): every
schedule, many iterations, exactly (the same FP64 formula)."""
import pytest

from ace_b200 import NNPError
from ace_b200.nnp import DECAY, decay_step
from oracle import ref


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref (compiled reference) not built")
@pytest.mark.parametrize("kind", sorted(DECAY))
def test_decay_matches_reference(kind):
    ref.lib()
    for alpha, period in ((1e-3, 5), (0.05, 7), (0.5, 3)):
        g, gr = 1e-2, 1e-2
        for step in range(40):
            g = decay_step(kind, alpha, period, g, step)
            gr = ref.lib().ref_decay_step(DECAY[kind], alpha, period, gr, step)
            assert g == gr, (kind, alpha, step)


def test_decay_errors():
    with pytest.raises(NNPError):
        decay_step(0, 0.1, 1, 1.0, 1)
    with pytest.raises(NNPError):
        decay_step("STEP", 0.1, 0, 1.0, 1)
