"""The committed Fortran interface (fortran/wql3d_c.f90) agrees with the C
header: the bind(C) descriptor types list the C struct fields in order, the
ABI version matches, and every interface names an exported entry point (no
Fortran compiler in this image, so the check is textual)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_fields(struct):
    src = open(os.path.join(ROOT, "include", "wql3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), src, flags=re.S).group(1)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        for part in decl.split(","):
            m = re.search(r"(\w+)\s*(\[\d+\])?\s*$", part.strip())
            names.append(m.group(1))
    return names


def _f_fields(typ):
    src = open(os.path.join(ROOT, "fortran", "wql3d_c.f90")).read()
    body = re.search(r"type, bind\(C\) :: %s\n(.*?)end type" % typ, src, flags=re.S).group(1)
    names = []
    for line in body.splitlines():
        if "::" not in line:
            continue
        for part in line.split("::")[1].split(","):
            names.append(re.sub(r"\(.*?\)", "", part).strip())
    return names


def test_descriptor_fields_match_the_header():
    assert [n.lower() for n in _f_fields("wql3d_block_desc")] == [n.lower() for n in _c_fields("wql3d_block_desc")]
    assert [n.lower() for n in _f_fields("wql3d_domain_desc")] == [n.lower() for n in _c_fields("wql3d_domain_desc")]


def test_abi_version_and_entry_points():
    src = open(os.path.join(ROOT, "fortran", "wql3d_c.f90")).read()
    hdr = open(os.path.join(ROOT, "include", "wql3d.h")).read()
    v = re.search(r"WQL3D_ABI_VERSION = (\d+)", src).group(1)
    assert "#define WQL3D_ABI_VERSION %s" % v in hdr
    names = set(re.findall(r"function (wql3d_\w+)\(", src))
    declared = set(re.findall(r"(wql3d_\w+)\s*\(", re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)))
    assert names and names <= declared
    for f in ("rk_vector_wql3d.f90", "time_step_wql3d.f90", "traditional_cartesian_rhs_wql3d.f90"):
        body = open(os.path.join(ROOT, "fortran", f)).read()
        for used in re.findall(r"(wql3d_\w+)\(", body):
            assert used in names, (f, used)
