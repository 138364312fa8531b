import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rust-simulation-tools_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def gpu_available() -> bool:
    try:
        import rust_simulation_tools as rst

        return rst.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def small_system(tmp_path_factory):
    """200 + 20 atom synthetic complex with 3 frames, written as prmtop + DCD."""
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("small")
    s = S.make_system(200, 20, seed=7)
    fr = S.make_frames(s, 3, seed=8)
    S.write_prmtop(s, str(d / "s.prmtop"))
    S.write_dcd(fr, str(d / "s.dcd"))
    return s, fr, str(d / "s.prmtop"), str(d / "s.dcd")
