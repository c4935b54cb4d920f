"""The step-solver adapter inside the reference's own main (schemi_b200/host/schemi_adapter).

``oracle/_ref/schemi_adapter_oracle`` is the reference solver compiled from its sources with one
more branch in its step-solver factory (src/interfaces/abstractStepSolver.cpp:78): the names
``Gpu<order>`` make ``gpuStepSolver``, which runs each step through the C-ABI of
include/fvstep.h.  Linked against the C-ABI over the CPU oracle (oracle/lib/
libschemi_fv_oracle.so), every deck fixture the reference wrote, with its approximation order X
renamed GpuX, must give the reference's files byte for byte: the adapter's deck reading,
upload, time-step hand-over and write-back into the phase (from which main's CFL block and
output writer work) are then exactly the reference step's.  The same binary linked against the
CUDA library is replayed by tests/test_gpu_adapter.py.
"""

import os
import subprocess

import pytest

from deck_replay import fixtures, replay, step_order

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER_ORACLE = os.path.join(ROOT, "oracle", "_ref", "schemi_adapter_oracle")

STEPPED = [n for n in fixtures() if step_order(n)]


def _binary():
    if not os.path.exists(ADAPTER_ORACLE):
        pytest.fail(f"{ADAPTER_ORACLE} is not built (make -C oracle ref)")
    return ADAPTER_ORACLE


def test_every_step_solver_has_fixtures():
    orders = {step_order(n) for n in STEPPED}
    assert {"SecondOrder", "SecondOrderRK", "ThirdOrderCada"} <= orders


@pytest.mark.parametrize("name", STEPPED)
def test_reference_main_with_adapter_matches_reference(tmp_path, name):
    problems = replay(_binary(), name, str(tmp_path), reference_main=True)
    assert not problems, "\n".join(problems)


def test_unknown_gpu_order_is_refused_by_the_factory(tmp_path):
    """A Gpu name that is not an order: the factory's own message, before any step or output."""
    from deck_replay import ORDER, load, unpack_inputs

    z = load("tube40_fresh")
    unpack_inputs(z, str(tmp_path))
    main_txt = ORDER.sub(rb"\1GpuFourthOrder\3", z["run0:main.txt"].tobytes())
    (tmp_path / "set" / "main.txt").write_bytes(main_txt)
    res = subprocess.run([_binary()], cwd=tmp_path, stdin=subprocess.DEVNULL, capture_output=True,
                         text=True, timeout=120)
    assert res.returncode != 0
    assert "Unknown gas dynamics approximation order." in res.stderr + res.stdout
    assert not (tmp_path / "result" / "output_000001.tsv").exists()


def test_deck_outside_the_step_is_refused_before_the_first_step(tmp_path):
    """A deck with turbulence: the adapter refuses at the factory, with the deck reader's message."""
    from deck_replay import ORDER, load, unpack_inputs

    z = load("tube40_fresh")
    unpack_inputs(z, str(tmp_path))
    main_txt = ORDER.sub(rb"\1Gpu\2\3", z["run0:main.txt"].tobytes())
    lines = main_txt.split(b"\n")
    i = lines.index(b"#Turbulence_flag")
    lines[i + 1] = b"on"
    (tmp_path / "set" / "main.txt").write_bytes(b"\n".join(lines))
    res = subprocess.run([_binary()], cwd=tmp_path, stdin=subprocess.DEVNULL, capture_output=True,
                         text=True, timeout=120)
    assert res.returncode != 0
    assert "turbulence models are not part of this step" in res.stderr + res.stdout
    assert not (tmp_path / "result" / "output_000001.tsv").exists()
