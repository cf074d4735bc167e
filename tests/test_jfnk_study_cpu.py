"""The Jacobian-free Newton-Krylov study on the oracle (oracle/jfnk_study.py)
stays runnable: 60 first-order iterations on the 1/16 plate, with the
Jacobian-free product and with the Picard matrix, both lower the residual
monitor below 0.5 of its maximum without blowing up."""
import pytest


@pytest.fixture(scope="module")
def study():
    import port
    if not port.available():
        pytest.skip("oracle/_ref/liboracle.so not built")
    import jfnk_study as s
    return s


def test_short_runs(study):
    out = {m: study.run("first", m, 60, 100.0, 16, 0) for m in ("picard", "jfnk")}
    for m, o in out.items():
        assert o["hist"] and o["hist"][-1][0] != "blowup", (m, o["hist"])
        assert o["hist"][-1][1] < 0.5, (m, o["hist"])
