"""Task-deck driver (schemi_b200/lib/fvrun) on the GPU against the reference solver's own files.

Each ``golden/deck_<name>.npz`` fixture is replayed in a fresh directory: the driver's
``result/output_<NNNNNN>.tsv``, ``result/Time.tsv``, ``fieldsOutput/output_<NNNNNN>/*.dat`` and
``timeOfCalculation.tsv`` must equal the reference's byte for byte, and the chemistry deck's
values to its stored relative tolerance (the chemistry pass agrees with the reference to
rounding; the driver also prints the total concentration as the sum of the species', where the
reference prints the 0.5 average of two totals), and the Redlich-Kwong and Kataoka decks to their
stored device tolerance (their cubic and Newton iterations use the device's transcendental
functions, and the cubic is solved in FP64 where the reference uses long double).
"""

import pytest

from deck_replay import fixtures, replay
from schemi_b200.build import DRIVER

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", fixtures())
def test_driver_matches_reference_files(tmp_path, name):
    problems = replay(DRIVER, name, str(tmp_path), gpu=True)
    assert not problems, "\n".join(problems)
