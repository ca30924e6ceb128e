"""The Mojo provider package source (dataframe_mojo_b200/mojo/dataframe_provider):
no Mojo toolchain exists here, so these checks read it as text -- it defines
exactly the thirteen functions dataframe/_accel_provider.mojo imports, every
C entry point it calls is declared in include/dfcuda.h and exported by the
library, and its dfc_timings mirror lists the header's fields in order."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "dataframe_mojo_b200" / "mojo" / "dataframe_provider"
HEADER = (ROOT / "include" / "dfcuda.h").read_text()

PROVIDER_FUNCTIONS = {
    "installed", "execute", "describe", "execute_profiled", "handoff_supports", "handoff_execute",
    "handoff_estimate", "devices", "transfer_model", "pipeline_supports", "pipeline_estimate",
    "pipeline_costs", "run_pipeline",
}


def sources() -> str:
    return "\n".join(p.read_text() for p in sorted(PKG.glob("*.mojo")))


def test_package_defines_the_thirteen_functions():
    init = (PKG / "__init__.mojo").read_text()
    public = {m for m in re.findall(r"^def ([a-z][a-z_]*)\(", init, re.M)}
    assert public == PROVIDER_FUNCTIONS


def test_called_entry_points_exist():
    from dataframe_mojo_b200 import _native as N

    called = set(re.findall(r'lib\.call\["(dfc_[a-z_]+)"', sources()))
    assert called, "no entry points found"
    declared = set(re.findall(r"^DFC_API [^(]*?\b(dfc_[a-z_]+)\(", HEADER, re.M))
    assert called <= declared, called - declared
    exported = {name for name, *_ in N.SIGNATURES}
    assert called <= exported, called - exported


def test_timings_mirror_matches_header():
    body = re.search(r"typedef struct dfc_timings \{(.*?)\} dfc_timings;", HEADER, re.S).group(1)
    header_fields = re.findall(r"^\s*\w+ (\w+);", body, re.M)
    mojo = re.search(r"struct DfcTimings\(.*?\):(.*?)@staticmethod", sources(), re.S).group(1)
    mojo_fields = re.findall(r"^\s*var (\w+):", mojo, re.M)
    assert mojo_fields == header_fields
