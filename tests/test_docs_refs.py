"""Every file of this repository that DESIGN.md, INTEGRATION.md or BASELINE.md
names in backticks exists (paths under tests/, oracle/, profiles/, include/,
cpu-ipc_b200/, and csrc/ for the library's sources), so the documents do not
point at files that were renamed or removed."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PREFIXES = ("tests/", "oracle/", "profiles/", "include/", "cpu-ipc_b200/", "csrc/")


@pytest.mark.parametrize("doc", ["DESIGN.md", "INTEGRATION.md", "BASELINE.md"])
def test_named_repository_files_exist(doc):
    text = open(os.path.join(ROOT, doc)).read()
    missing = []
    for path in re.findall(r"`([A-Za-z0-9_./-]+)`", text):
        if not path.startswith(PREFIXES) or "*" in path:
            continue
        full = os.path.join(ROOT, "cpu-ipc_b200", path) if path.startswith("csrc/") else os.path.join(ROOT, path)
        if not os.path.exists(full.rstrip("/")):
            missing.append(path)
    assert not missing, missing
