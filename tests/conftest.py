import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _load_package():
    if "compactles_b200" in sys.modules:
        return sys.modules["compactles_b200"]
    pkg = ROOT / "compactles.jl_b200"
    spec = importlib.util.spec_from_file_location(
        "compactles_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["compactles_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_package()
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running oracle validation case")


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    # parity figures that tests recorded beside their asserted bounds, so a
    # quiet run still shows them
    parity = sys.modules.get("parity")
    if parity is not None and parity.LINES:
        terminalreporter.section("parity figures")
        for ln in parity.LINES:
            terminalreporter.write_line(ln)
