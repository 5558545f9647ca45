"""A stand-in for the h5py calls the transport makes, for hosts without
h5py (test infrastructure only).

It keeps the datasets of one "HDF5" file in a NumPy .npz archive at that
path: ``File(path, "x")`` creates it on close, ``File(path, "r")`` reads
it; ``create_dataset(name, data=...)`` and ``handle[name]`` (with
``.shape``, ``.dtype`` and ``[...]``) are all the transport uses.  Files
written with it are not HDF5 files.
"""
import os

import numpy as np

__version__ = "stub"


def _key(name):
    return name.lstrip("/").replace("/", "__")


class _Dataset:
    def __init__(self, array):
        self._a = array
        self.shape = array.shape
        self.dtype = array.dtype

    def __getitem__(self, item):
        return self._a[item]


class File:
    def __init__(self, path, mode="r"):
        self.path = os.fspath(path)
        self.mode = mode
        if mode == "r":
            with np.load(self.path, allow_pickle=False) as z:
                self._data = {k: z[k] for k in z.files}
        elif mode == "x":
            if os.path.exists(self.path):
                raise FileExistsError(self.path)
            self._data = {}
        else:
            raise ValueError(f"mode {mode!r} is not supported by the stand-in")

    def create_dataset(self, name, data):
        key = _key(name)
        if key in self._data:
            raise ValueError(f"dataset {name} exists")
        self._data[key] = np.array(data)
        return _Dataset(self._data[key])

    def __getitem__(self, name):
        return _Dataset(self._data[_key(name)])

    def close(self):
        if self.mode == "x" and self._data is not None:
            with open(self.path, "xb") as f:
                np.savez(f, **self._data)
            self._data = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False
