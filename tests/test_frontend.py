"""Text front-end (system text -> step body) against the reference's own output.

tests/golden/codegen_cases.json was generated by running the reference's sysparse.cpp +
codegen.cpp (compiled as-is into oracle/_ref, see tests/golden/make_golden.py) on the
library presets and on synthetic edge cases; the engine's front-end must produce the
same variables, parameters and step bodies byte for byte, and fail where it fails."""
import pytest

import ucb
from helpers import codegen_cases

SCHEMES = ["Euler", "Euler-Cromer", "Explicit Midpoint", "RK4", "DOPRI78", "CD"]


@pytest.mark.parametrize("name", sorted(codegen_cases()))
def test_codegen_matches_reference(name):
    c = codegen_cases()[name]
    for sc in SCHEMES:
        ref = c["schemes"][sc]
        if ref.startswith("@ERROR"):
            with pytest.raises(ucb.UcbError):
                ucb.codegen(c["text"], c["alphabet"], sc, c["order"] == "system", c["funcs"])
            continue
        body, vs, ps = ucb.codegen(c["text"], c["alphabet"], sc, c["order"] == "system", c["funcs"])
        assert vs == c["vars"]
        assert ps == c["params"]
        assert body == ref, f"{name}/{sc}"
