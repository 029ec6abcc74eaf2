"""The reference's twelve AFR unit cases through the reference's own C++ operation API and
payload types, with the engine plugged in as the strategy (include/umpalumpa_fr_afr.hpp).

The program (tests/cpp/fr_afr_cases.cpp) is built where the reference sources are present
(tests/cpp/Makefile, run by __graft_entry__.build()) and travels as a built file."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_bin", "fr_afr_cases")
# written by the build when no reference checkout was present to build the program from
NO_REFERENCE_MARK = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_bin", "NO_REFERENCE")


def test_reference_unit_cases_through_reference_api(cuda):
    if not os.path.exists(BIN):
        if os.path.exists(NO_REFERENCE_MARK):
            pytest.skip("built without a reference checkout: " + open(NO_REFERENCE_MARK).read().strip())
        pytest.fail("the reference-API test program is missing although the build had the reference "
                    "checkout (tests/_bin/fr_afr_cases; run __graft_entry__.build())")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 12
