"""The Fortran iso_c_binding module (include/diablo_gpu.f90) against the C
header, parsed on the CPU (there is no Fortran compiler on this image, so
the parse is the check):

- every function the header declares is bound under its C name, and nothing
  else is;
- each binding takes as many arguments as the C prototype, with a matching
  interoperable kind and passing mode (C scalars by value; pointers as
  type(c_ptr) by value or as Fortran arguments by reference);
- type(diablo_params) has the C struct's fields in the same order, with the
  same kinds and array lengths;
- the integer constants equal the header's enum values.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diablo_gpu.h")
MODULE = os.path.join(ROOT, "include", "diablo_gpu.f90")


def _fortran_lines():
    out, cur = [], ""
    for raw in open(MODULE):
        line = raw.split("!")[0].rstrip()
        if not line.strip():
            continue
        if cur:
            line = cur + " " + line.strip()
            cur = ""
        if line.endswith("&"):
            cur = line[:-1].rstrip()
            continue
        out.append(line.strip())
    assert not cur
    return out


def _c_source():
    src = open(HEADER).read()
    return re.sub(r"/\*.*?\*/", "", src, flags=re.S)


def _c_prototypes():
    src = _c_source()
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w \*]*?)\b(diablo_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", src):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        params = [] if args in ("", "void") else [a.strip() for a in args.split(",")]
        protos[name] = (ret, params)
    return protos


def _fortran_interfaces():
    lines = _fortran_lines()
    funcs, cur = {}, None
    for line in lines:
        m = re.match(r'function (\w+)\(([^)]*)\) bind\(C, name="(\w+)"\)', line)
        if m:
            assert m.group(1) == m.group(3), line
            args = [a.strip() for a in m.group(2).split(",") if a.strip()]
            cur = {"name": m.group(1), "args": args, "decl": {}}
            continue
        if cur is None:
            continue
        if re.match(r"end function (\w+)", line):
            assert line.split()[-1] == cur["name"]
            funcs[cur["name"]] = cur
            cur = None
            continue
        m = re.match(r"(type\(c_ptr\)|type\(diablo_params\)|integer\(c_int\)|integer\(c_long_long\)|"
                     r"real\(c_double\))((?:, *[a-z]+(?:\([a-z]+\))?)*) *:: *(.+)$", line)
        if m:
            kind, attrs = m.group(1), m.group(2)
            for var in re.split(r",\s*(?![^(]*\))", m.group(3)):
                vm = re.match(r"(\w+)(\([^)]*\))?", var.strip())
                cur["decl"][vm.group(1)] = (kind, "value" in attrs, vm.group(2))
    assert cur is None
    return funcs


C_SCALAR = {"int": "integer(c_int)", "double": "real(c_double)", "long long": "integer(c_long_long)"}


def test_every_declared_function_is_bound_once():
    assert sorted(_fortran_interfaces()) == sorted(_c_prototypes())


def test_arguments_match_the_prototypes():
    protos, funcs = _c_prototypes(), _fortran_interfaces()
    for name, (ret, params) in protos.items():
        f = funcs[name]
        assert len(f["args"]) == len(params), name
        # result kind
        rk = f["decl"][name][0]
        if "*" in ret:
            assert rk == "type(c_ptr)", name
        else:
            assert rk == C_SCALAR[ret.replace("const", "").strip()], name
        for arg, cp in zip(f["args"], params):
            kind, by_value, dims = f["decl"][arg]
            ctype = re.sub(r"\b(const)\b", "", cp).strip()
            ctype = ctype[: ctype.rfind(" ")].strip() if " " in ctype else ctype
            if "*" in cp:
                if by_value:
                    assert kind == "type(c_ptr)", (name, arg)
                else:
                    base = " ".join(re.sub(r"\bconst\b|\*", " ", cp).split()[:-1])
                    if cp.count("*") == 2:          # array of pointers
                        assert kind == "type(c_ptr)" and dims, (name, arg)
                    elif base == "diablo_params":
                        assert kind == "type(diablo_params)", (name, arg)
                    else:
                        assert kind == C_SCALAR[base], (name, arg)
            else:
                assert by_value and kind == C_SCALAR[ctype], (name, arg, cp)


def _c_struct_fields():
    src = _c_source()
    body = re.search(r"typedef struct diablo_params \{(.*?)\} diablo_params;", src, re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(int|double)\s+(.*)$", decl, re.S)
        kind = C_SCALAR[m.group(1)]
        for var in m.group(2).split(","):
            vm = re.match(r"\s*(\w+)(?:\[(\w+)\])?", var)
            n = 8 if vm.group(2) == "DIABLO_MAX_TH" else 1
            fields.append((vm.group(1), kind, n))
    return fields


def _fortran_type_fields():
    lines = _fortran_lines()
    i = lines.index("type, bind(C) :: diablo_params")
    fields = []
    for line in lines[i + 1:]:
        if line.startswith("end type"):
            break
        kind, rest = line.split("::")
        for var in re.split(r",\s*(?![^(]*\))", rest):
            vm = re.match(r"\s*(\w+)(?:\((\w+)\))?", var)
            n = 8 if vm.group(2) == "DIABLO_MAX_TH" else 1
            fields.append((vm.group(1), kind.strip(), n))
    return fields


def test_params_type_matches_the_c_struct():
    assert _fortran_type_fields() == _c_struct_fields()


def test_constants_match_the_header():
    src = _c_source()
    cvals = {}
    for body in re.findall(r"enum \w+ \{(.*?)\};", src, re.S):
        for item in body.split(","):
            m = re.match(r"\s*(DIABLO_\w+)\s*=\s*(-?\d+)", item)
            if m:
                cvals[m.group(1)] = int(m.group(2))
    for m in re.finditer(r"#define (DIABLO_ABI_VERSION|DIABLO_MAX_TH) (\d+)", src):
        cvals[m.group(1)] = int(m.group(2))
    fvals = {}
    for line in _fortran_lines():
        m = re.match(r"integer\(c_int\), parameter :: (DIABLO_\w+) = (-?\d+)$", line)
        if m:
            fvals[m.group(1)] = int(m.group(2))
    assert fvals, "no constants parsed"
    for k, v in fvals.items():
        assert cvals[k] == v, k
    for k in ("DIABLO_OK", "DIABLO_ERR_TIMEOUT", "DIABLO_MIXED", "DIABLO_TH", "DIABLO_LAYOUT_PHYSICAL"):
        assert k in fvals, k


def test_module_structure_is_balanced():
    lines = _fortran_lines()
    assert lines[0] == "module diablo_gpu" and lines[-1] == "end module diablo_gpu"
    assert sum(l == "interface" for l in lines) == sum(l == "end interface" for l in lines) == 1
    n_fun = sum(bool(re.match(r"function \w+\(", l)) for l in lines)
    n_end = sum(bool(re.match(r"end function \w+", l)) for l in lines)
    assert n_fun == n_end
