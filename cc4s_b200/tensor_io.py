"""cc4s tensor files: a YAML header and a dense ``.elements`` file.

Restates the format of the reference's ``TensorIo`` (src/main/TensorIo.cxx:
``read``/``readTensor`` 142-247, the element readers 340-499, ``writeTensor``
109-158): the header holds ``version``, ``scalarType`` (``Real64`` or
``Complex64``), ``dimensions`` (per dimension ``length`` and an optional
``type`` such as ``State``), ``elements.type`` (``TextFile``: one number per
line, complex numbers as ``(re,im)``; ``IeeeBinaryFile``: raw little-endian
values), ``unit`` and optional ``metaData``.  Elements are stored with the
first index fastest (column-major).  Block-sparse files (``nonZeroCondition``)
are rejected.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
import yaml

VERSION = 100
SCALAR_TYPES = {"Real64": np.float64, "Complex64": np.complex128}


@dataclass
class Tensor:
    """A tensor read from or written to a cc4s tensor file."""
    values: np.ndarray                    # dims in file order (column-major on disk)
    dimension_types: list = field(default_factory=list)
    unit: float = 1.0
    meta_data: dict = field(default_factory=dict)


def _elements_path(yaml_path):
    base = yaml_path[:-5] if yaml_path.endswith(".yaml") else yaml_path
    return base + ".elements"


def _parse_text_number(token, complex_values):
    token = token.strip()
    if token.startswith("("):
        re_, im_ = token[1:-1].split(",")
        return complex(float(re_), float(im_))
    v = float(token)
    return complex(v, 0.0) if complex_values else v


def read(yaml_path):
    """Reads a cc4s tensor file (header ``*.yaml`` and ``*.elements``)."""
    with open(yaml_path) as f:
        node = yaml.safe_load(f)
    if not isinstance(node, dict):
        raise ValueError("%s: not a tensor header" % yaml_path)
    version = int(node.get("version", -1))
    if version != VERSION:
        raise ValueError("%s: serialization version %d, expecting %d" % (yaml_path, version, VERSION))
    scalar = node.get("scalarType")
    if scalar not in SCALAR_TYPES:
        raise ValueError("%s: unsupported scalarType %r" % (yaml_path, scalar))
    if node.get("nonZeroCondition"):
        raise ValueError("%s: block-sparse tensors are not supported" % yaml_path)
    dims = node.get("dimensions") or {}
    keys = sorted(dims, key=lambda k: int(k))
    lens = [int(dims[k]["length"]) for k in keys]
    types = [dims[k].get("type") for k in keys]
    dtype = SCALAR_TYPES[scalar]
    count = int(np.prod(lens)) if lens else 1
    etype = (node.get("elements") or {}).get("type")
    path = _elements_path(yaml_path)
    if etype == "IeeeBinaryFile":
        flat = np.fromfile(path, dtype=np.dtype(dtype).newbyteorder("<"), count=count)
    elif etype == "TextFile":
        with open(path) as f:
            tokens = [t for t in (line.strip() for line in f) if t and not t.startswith("#")]
        flat = np.array([_parse_text_number(t, dtype is np.complex128) for t in tokens[:count]],
                        dtype=dtype)
    else:
        raise ValueError("%s: unknown elements type %r" % (yaml_path, etype))
    if flat.size != count:
        raise ValueError("%s: %d elements, expecting %d" % (path, flat.size, count))
    values = flat.reshape(lens, order="F") if lens else flat.reshape(())
    return Tensor(values=values, dimension_types=types, unit=float(node.get("unit", 1.0)),
                  meta_data=node.get("metaData") or {})


def write(yaml_path, tensor, binary=True):
    """Writes a cc4s tensor file (header and elements) from a Tensor."""
    values = np.asarray(tensor.values)
    cplx = np.iscomplexobj(values)
    dims = {}
    for d, n in enumerate(values.shape):
        entry = {"length": int(n)}
        if d < len(tensor.dimension_types) and tensor.dimension_types[d]:
            entry["type"] = tensor.dimension_types[d]
        dims[d] = entry
    header = {"type": "Tensor", "scalarType": "Complex64" if cplx else "Real64",
              "version": VERSION, "dimensions": dims,
              "elements": {"type": "IeeeBinaryFile" if binary else "TextFile"},
              "unit": float(tensor.unit), "metaData": tensor.meta_data or {}}
    with open(yaml_path, "w") as f:
        yaml.safe_dump(header, f, sort_keys=False)
    flat = values.reshape(-1, order="F")
    path = _elements_path(yaml_path)
    if binary:
        flat.astype(np.complex128 if cplx else np.float64).astype(
            np.dtype(np.complex128 if cplx else np.float64).newbyteorder("<")).tofile(path)
    else:
        with open(path, "w") as f:
            for v in flat:
                f.write("(%.17g,%.17g)\n" % (v.real, v.imag) if cplx else "%.17g\n" % v)
    return os.path.abspath(yaml_path)
