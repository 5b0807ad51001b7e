"""Model and structure files.

Models are stored in the reference's BaseIO JSON format
(bindings/rascal/utils/io.py:16-470), so a model fitted with the reference
(for instance its `simple_gap_model.json`) loads here and a model saved here
loads in the reference:

* every object is a dict {version: "0.1", class_name, module_name,
  init_params, data}, nested objects serialised the same way;
* numpy arrays become ["npy", list], or, above 50 MB, a side file
  `<file>-<class>-<key>.npy` named in the JSON;
* dict keys that read as integers (the self contributions per atomic
  number) are integers again after loading.

The module and class names written are the reference's
(`rascal.models.krr.KRR` and so on); loading maps them to this package's
classes.

Structures are read from the ASE-db JSON layout that the reference's
`ManagerCollection.add_structures(filename)` reads
(structure_managers/structure_manager_collection.hh:225-256) and from
extended XYZ (the `Lattice=`, `Properties=`, `pbc=` header the reference's
test data uses). Both give the frame dicts that `AtomsList` takes.
"""
import json
import os
import re
import shlex

import numpy as np

VERSION = "0.1"
_LARGE = 50e6

# (reference module, class) <-> this package's class
_REGISTRY = {
    ("rascal.models.krr", "KRR"): ("librascal_b200.models", "KRR"),
    ("rascal.models.kernels", "Kernel"): ("librascal_b200.models", "Kernel"),
    ("rascal.models.sparse_points", "SparsePoints"): ("librascal_b200.models", "SparsePoints"),
    ("rascal.representations.spherical_invariants", "SphericalInvariants"):
        ("librascal_b200.representations", "SphericalInvariants"),
    ("rascal.representations.spherical_expansion", "SphericalExpansion"):
        ("librascal_b200.representations", "SphericalExpansion"),
}
_REFERENCE_NAME = {v: k for k, v in _REGISTRY.items()}
_KEYS = ("version", "class_name", "module_name", "init_params", "data")


def _class(module_name, class_name):
    import importlib
    mod, cls = _REGISTRY.get((module_name, class_name), (module_name, class_name))
    if not mod.startswith("librascal_b200"):
        raise RuntimeError("cannot load objects of class %s.%s" % (module_name, class_name))
    return getattr(importlib.import_module(mod), cls)


def _is_serialisable(obj):
    return all(hasattr(obj, m) for m in ("_get_init_params", "_get_data", "_set_data"))


def _is_object_dict(d):
    return isinstance(d, dict) and all(k in d for k in _KEYS)


def to_dict(obj, depth=0):
    """The BaseIO dict of `obj` (nested objects included)."""
    if depth >= 20:
        raise ValueError("more than 20 levels of nested objects: circular reference?")
    if not _is_serialisable(obj):
        raise ValueError('input object: "{}" does not implement the serialisation interface'.format(obj))
    state = dict(init_params=dict(obj._get_init_params()), data=dict(obj._get_data()))
    for part in state.values():
        for k, v in part.items():
            if _is_serialisable(v):
                part[k] = to_dict(v, depth + 1)
            elif isinstance(v, list):
                part[k] = [to_dict(x, depth + 1) if _is_serialisable(x) else x for x in v]
    mod, cls = _REFERENCE_NAME.get((type(obj).__module__, type(obj).__name__),
                                   (type(obj).__module__, type(obj).__name__))
    return dict(version=VERSION, class_name=cls, module_name=mod, init_params=state["init_params"],
                data=state["data"])


def from_dict(d):
    """The object described by a BaseIO dict."""
    if d.get("version") != VERSION:
        raise RuntimeError("unsupported serialisation version: {}".format(d.get("version")))
    parts = {}
    for name in ("init_params", "data"):
        parts[name] = {}
        for k, v in d[name].items():
            if _is_object_dict(v):
                v = from_dict(v)
            elif isinstance(v, list):
                v = [from_dict(x) if _is_object_dict(x) else x for x in v]
            parts[name][k] = v
    obj = _class(d["module_name"], d["class_name"])(**parts["init_params"])
    obj._set_data(parts["data"])
    return obj


def _int_keys(o):
    return {(int(k) if isinstance(k, str) and re.fullmatch(r"-?\d+", k) else k): v for k, v in o.items()}


def _arrays_out(fn, d, class_name):
    base = os.path.splitext(fn)[0]
    for k, v in list(d.items()):
        if isinstance(v, dict):
            _arrays_out(fn, v, v["class_name"].lower() if "class_name" in v else class_name)
        elif isinstance(v, np.ndarray):
            if v.nbytes > _LARGE:
                side = base + "-{}-{}.npy".format(class_name, k)
                np.save(side, v)
                d[k] = os.path.basename(side)
            else:
                d[k] = ["npy", v.tolist()]


def _arrays_in(d, path):
    for k, v in list(d.items()):
        if isinstance(v, dict):
            _arrays_in(v, path)
        elif isinstance(v, str) and v.endswith(".npy"):
            d[k] = np.load(os.path.join(path, v), mmap_mode="r")
        elif isinstance(v, list) and len(v) == 2 and isinstance(v[0], str) and v[0] == "npy":
            d[k] = np.array(v[1])


def dump_obj(fn, obj):
    """Save `obj` (KRR, Kernel, SparsePoints, a representation) as JSON."""
    fn = os.path.abspath(fn)
    if os.path.splitext(fn)[1] != ".json":
        raise NotImplementedError("Unknown file extention: {}".format(os.path.splitext(fn)[1]))
    d = to_dict(obj)
    _arrays_out(fn, d, d["class_name"].lower())
    with open(fn, "w") as f:
        json.dump(d, f, sort_keys=True, indent=2)


def load_obj(fn):
    """Load an object saved by dump_obj here or by the reference."""
    fn = os.path.abspath(fn)
    if os.path.splitext(fn)[1] != ".json":
        raise NotImplementedError("Unknown file extention: {}".format(os.path.splitext(fn)[1]))
    with open(fn) as f:
        d = json.load(f, object_hook=_int_keys)
    if not _is_object_dict(d):
        raise RuntimeError("The file: {}; does not contain a valid dictionary representation of an "
                           "object.".format(fn))
    _arrays_in(d, os.path.dirname(fn))
    return from_dict(d)


# ------------------------------------------------------------------ structures
def read_ase_json(fn, start=0, length=None):
    """Frames of an ASE-db JSON file, sorted by id; `start` and `length`
    select a range as in ManagerCollection.add_structures."""
    with open(fn) as f:
        d = json.load(f)
    if not isinstance(d, dict) or "ids" not in d:
        raise RuntimeError("The json structure format is not recognized")
    ids = sorted(int(i) for i in d["ids"])[start:]
    if length is not None and length >= 0:
        ids = ids[:length]
    frames = []
    for i in ids:
        e = d[str(i)]
        frames.append(dict(positions=np.asarray(e["positions"], float),
                           numbers=np.asarray(e["numbers"], np.int32),
                           cell=np.asarray(e.get("cell", np.zeros((3, 3))), float).reshape(3, 3),
                           pbc=np.asarray(e.get("pbc", [False] * 3), bool).reshape(3)))
    return frames


_SYMBOLS = ("X H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se "
            "Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho "
            "Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es "
            "Fm Md No Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()
_NUMBER = {s: z for z, s in enumerate(_SYMBOLS)}


def _value(text):
    t = text.strip()
    if t in ("T", "True"):
        return True
    if t in ("F", "False"):
        return False
    for cast in (int, float):
        try:
            return cast(t)
        except ValueError:
            pass
    parts = t.split()
    if len(parts) > 1:
        vals = [_value(p) for p in parts]
        if all(isinstance(v, (bool, np.bool_)) for v in vals):
            return np.array(vals, bool)
        if all(isinstance(v, (int, float)) for v in vals):
            return np.array(vals, float)
    return t


def read_extxyz(fn, index=":"):
    """Frames of an extended XYZ file (`index` a Python slice string such as
    ":100", or an int). Each frame is a dict with positions, numbers, cell
    (rows are lattice vectors; zeros without a Lattice), pbc, `info` (the
    header's other key=value pairs, e.g. energy) and `arrays` (the other
    per-atom columns, e.g. force)."""
    frames = []
    with open(fn) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        n = int(lines[i].split()[0])
        header = lines[i + 1]
        rows = [ln.split() for ln in lines[i + 2:i + 2 + n]]
        i += 2 + n
        info = {}
        for tok in shlex.split(header):
            if "=" in tok:
                k, v = tok.split("=", 1)
                info[k] = v
        props = info.pop("Properties", "species:S:1:pos:R:3").split(":")
        cols, c = {}, 0
        for name, kind, width in zip(props[0::3], props[1::3], props[2::3]):
            w = int(width)
            cols[name] = (kind, c, w)
            c += w
        arrays = {}
        for name, (kind, c0, w) in cols.items():
            block = [r[c0:c0 + w] for r in rows]
            if kind == "R":
                a = np.array(block, float)
            elif kind == "I":
                a = np.array(block, int)
            elif kind == "L":
                a = np.array([[x in ("T", "True") for x in b] for b in block])
            else:
                a = np.array(block, dtype=object)
            arrays[name] = a[:, 0] if w == 1 else a
        if "species" in arrays:
            numbers = np.array([_NUMBER[s] for s in arrays.pop("species")], np.int32)
        else:
            numbers = np.asarray(arrays.pop("Z"), np.int32)
        positions = np.asarray(arrays.pop("pos"), float)
        cell = np.zeros((3, 3))
        if "Lattice" in info:
            cell = np.array(info.pop("Lattice").split(), float).reshape(3, 3)
        pbc = np.array([cell.any()] * 3)
        if "pbc" in info:
            pbc = np.array([t in ("T", "True") for t in info.pop("pbc").split()])
        frames.append(dict(positions=positions, numbers=numbers, cell=cell, pbc=pbc,
                           info={k: _value(v) for k, v in info.items()}, arrays=arrays))
    if isinstance(index, int):
        return frames[index]
    a, b, s = (index.split(":") + [""] * 3)[:3]
    return frames[slice(int(a) if a else None, int(b) if b else None, int(s) if s else None)]
