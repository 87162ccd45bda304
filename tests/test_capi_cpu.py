"""C ABI checks that need no GPU: the library builds/loads, exports every
symbol include/pinyb200.h declares, and its system struct has the layout the
header defines."""
import ctypes as C
import os
import re

from piny_b200 import lib

HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "include", "pinyb200.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pinyb200_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_header_symbols():
    L = lib.load()
    names = header_functions()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(lib.EXPORTS)


def test_system_struct_layout_matches_oracle():
    from oracle.oracle import OrcEnergies, OrcSystem
    assert [f[0] for f in lib.PinySystem._fields_] == [f[0] for f in OrcSystem._fields_]
    assert C.sizeof(lib.PinySystem) == C.sizeof(OrcSystem)
    assert C.sizeof(lib.PinyEnergies) == C.sizeof(OrcEnergies)


def test_header_struct_fields_in_order():
    text = open(HEADER).read()
    body = text[text.index("typedef struct pinyb200_system"):text.index("} pinyb200_system;")]
    fields = []
    for line in body.splitlines()[1:]:
        line = line.split("/*")[0].strip().rstrip(";")
        if not line:
            continue
        decl = line.replace("const ", "").replace("*", " ")
        parts = decl.replace(",", " ").split()
        fields.extend(parts[1:])
    assert fields == [f[0] for f in lib.PinySystem._fields_]


def test_version_without_device():
    L = lib.load()
    assert L.pinyb200_version() == 1


def test_count_scratch_limits_match_header():
    text = open(HEADER).read()
    assert int(re.search(r"PINYB200_COUNT_MAX_ATOMS\s*=\s*(\d+)", text).group(1)) == lib.COUNT_MAX_ATOMS
    assert int(re.search(r"PINYB200_COUNT_MAX_PAIR_TYPES\s*=\s*(\d+)", text).group(1)) == lib.COUNT_MAX_PAIR_TYPES
