"""pytest configuration: the ``gpu`` marker, and the repository root on sys.path."""
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))




def load_package():
    """Imports the vexelray-sim-fluid_b200/ package (its directory name is not an identifier) as ``vexfluid``."""
    import importlib.util
    if "vexfluid" in sys.modules:
        return sys.modules["vexfluid"]
    pkg = ROOT / "vexelray-sim-fluid_b200"
    spec = importlib.util.spec_from_file_location("vexfluid", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vexfluid"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); runs through the C-ABI library")
