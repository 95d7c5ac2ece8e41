"""Source rules that the chained (programmatic dependent) launches rely on, checked on the CPU.

Every kernel is launched with programmatic stream serialisation, so the next kernel in a stream
may start before its predecessor has finished. That is only correct because each kernel's first
statement is grid_entry() (griddepcontrol.wait before any global memory access) and because every
launch goes through launch_k. A kernel added without either would race with its neighbours, so
these tests read the CUDA sources and fail on such a kernel.
"""
import re
from pathlib import Path

CSRC = Path(__file__).resolve().parents[1] / "dmrjtensor.jl_b200" / "csrc"


def kernel_bodies():
    """(file, kernel name, first statement of the body) for every __global__ function."""
    out = []
    for f in sorted(CSRC.glob("*.cu")):
        src = f.read_text()
        for m in re.finditer(r"__global__", src):
            brace = src.index("{", m.end())
            head = src[m.end():brace]
            name = re.findall(r"(\w+)\s*\(", head)
            name = name[-1] if name else "?"
            body = src[brace + 1:]
            first = body.lstrip().split(";", 1)[0].strip()
            out.append((f.name, name, first))
    return out


def test_every_kernel_starts_with_grid_entry():
    ks = kernel_bodies()
    assert len(ks) >= 30
    bad = [(f, n) for f, n, first in ks if first != "grid_entry()"]
    assert not bad, f"kernels whose first statement is not grid_entry(): {bad}"


def test_no_triple_chevron_launches():
    for f in sorted(CSRC.glob("*.cu")):
        assert "<<<" not in f.read_text(), f"{f.name} launches without launch_k"


def test_launch_helper_sets_programmatic_serialisation():
    src = (CSRC / "launch.cuh").read_text()
    assert "cudaLaunchAttributeProgrammaticStreamSerialization" in src
    wait = src.index("griddepcontrol.wait")
    trigger = src.index("griddepcontrol.launch_dependents")
    assert wait < trigger, "the trigger must come after the wait"
