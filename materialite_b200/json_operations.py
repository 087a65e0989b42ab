# Portions of this file restate the interface and the JSON document layout of materialite's
# materialite/json_operations.py: Copyright 2025 United States Government as represented by the Administrator
# of the National Aeronautics and Space Administration.  All Rights Reserved.  Licensed
# under the Apache License, Version 2.0 (http://www.apache.org/licenses/LICENSE-2.0);
# distributed on an "AS IS" BASIS, WITHOUT WARRANTIES OR CONDITIONS OF ANY KIND.

"""JSON persistence of a Material, in the layout of materialite/json_operations.py:23-122,
so that files move between this package and the reference: a "metadata" entry (origin,
dimensions, spacing), an optional "state", "regional_fields" by region label, and one
entry per point field.  Arrays are stored as {"data": ...}; tensors add their class name
and dimension string, orientations their class name."""

import gzip
import json

import numpy as np
import pandas as pd

from . import tensor as _tensor
from .material import Material
from .tensor import Orientation, Tensor

COORDINATE_LABELS = ("x", "y", "z", "x_id", "y_id", "z_id")


class MaterialEncoder(json.JSONEncoder):
    def default(self, obj):
        if isinstance(obj, Tensor):
            return {"data": np.asarray(obj.components).tolist(), "type": type(obj).__name__,
                    "dims": obj.dims_str}
        if isinstance(obj, Orientation):
            return {"data": np.asarray(obj.rotation_matrix).tolist(), "type": "Orientation"}
        if isinstance(obj, (np.number, np.ndarray)):
            return {"data": obj.tolist()}
        return super().default(obj)


def decoder_object_hook(dct):
    data = dct.get("data", None)
    if data is None:
        return dct
    kind = dct.get("type", None)
    if kind is None:
        return data
    cls = getattr(_tensor, kind)
    dims = dct.get("dims", None)
    return cls(np.asarray(data)) if dims is None else cls(np.asarray(data), dims)


def write_to_json(material, filename, compress=False):
    doc = {"metadata": {"origin": material.origin.tolist(),
                        "dimensions": material.dimensions.tolist(),
                        "spacing": material.spacing.tolist()}}
    if material.state:
        doc["state"] = material.state
    if material._regional_fields:
        doc["regional_fields"] = {}
        for region in material._regional_fields:
            labels = list(material.extract_regional_field(region).columns)
            doc["regional_fields"][region] = {
                label: material.extract_regional_field(region, label) for label in labels}
    for label in material._fields:
        if label not in COORDINATE_LABELS:
            doc[label] = material.extract(label)
    text = json.dumps(doc, cls=MaterialEncoder)
    if compress:
        with open(filename, "wb") as f:
            f.write(gzip.compress(text.encode("utf-8")))
    else:
        with open(filename, "w") as f:
            f.write(text)


def read_from_json(filename, decompress=False):
    if decompress:
        with open(filename, "rb") as f:
            text = gzip.decompress(f.read()).decode("utf-8")
    else:
        with open(filename) as f:
            text = f.read()
    doc = json.loads(text, object_hook=decoder_object_hook)
    meta = doc.pop("metadata")
    state = doc.pop("state", {})
    regional = doc.pop("regional_fields", {})
    material = Material(dimensions=meta["dimensions"], origin=meta["origin"],
                        spacing=meta["spacing"])
    if doc:
        material = material.create_fields(doc)
    material.state = state
    for region, columns in regional.items():
        material = material.create_regional_fields(region, pd.DataFrame(
            {k: (list(v) if isinstance(v, (Tensor, Orientation)) else v)
             for k, v in columns.items()}))
    return material
