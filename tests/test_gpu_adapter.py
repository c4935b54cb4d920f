"""The reference's own main with its step on the B200 library (drop-in check).

``oracle/_ref/schemi_adapter_gpu`` is the reference solver compiled from its sources with the
step-solver adapter (schemi_b200/host/schemi_adapter) registered in its factory under the names
``Gpu<order>``, linked against schemi_b200/lib/libschemi_fv.so.  Every deck fixture, with its
approximation order X renamed GpuX, runs the reference's task-file reader, CFL block and output
writer unchanged with each step on the GPU, and must give the reference's files: byte for byte,
or within the fixture's GPU tolerance (the real-gas mixtures, whose transcendental functions round
differently on the device) and the chemistry fixture's tolerance.
"""

import os

import pytest

from deck_replay import fixtures, replay, step_order

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER_GPU = os.path.join(ROOT, "oracle", "_ref", "schemi_adapter_gpu")

STEPPED = [n for n in fixtures() if step_order(n)]


@pytest.mark.gpu
@pytest.mark.parametrize("name", STEPPED)
def test_reference_main_on_the_gpu_library_matches_reference(tmp_path, name):
    if not os.path.exists(ADAPTER_GPU):
        pytest.fail(f"{ADAPTER_GPU} is not built (make -C oracle ref, after the CUDA library)")
    problems = replay(ADAPTER_GPU, name, str(tmp_path), gpu=True, reference_main=True)
    assert not problems, "\n".join(problems)
