"""Writes oracle_states.json: the oracle's (the C++ restatement's) results for the scenarios of
cases.py. Run from the repository root: python tests/golden/make_golden.py
The device must reproduce these bit for bit (tests/test_golden.py)."""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from conftest import ORACLE_EXTRA, build_oracle  # noqa: E402
from milldynamics3_b200 import capi  # noqa: E402
from milldynamics3_b200.sim import Backend  # noqa: E402

import cases  # noqa: E402


def main():
    b = Backend(capi.Lib(build_oracle(), "or_", ORACLE_EXTRA))
    out = {}
    for name in cases.cases():
        out[name] = cases.run_case(b, name)
        print(name, out[name], flush=True)
    with open(os.path.join(HERE, "oracle_states.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
