"""``Molecule``: the reference's molecule container (fml/fml.py:44-132).

Keeps the reference's attributes and method names. Descriptor generation
runs on the GPU through the batched kernels with a batch of one; for many
molecules use ``fml_b200.generate_coulomb_matrices`` /
``generate_arad_descriptors`` directly (one launch for the whole batch).
"""

import numpy as np

from .data import NUCLEAR_CHARGE
from .descriptors import (generate_arad_descriptors, generate_coulomb_matrices,
                          generate_local_coulomb_matrices, generate_unsorted_coulomb_matrices)


class Molecule:
    def __init__(self):
        self.natoms = -1
        self.energy = float("nan")
        self.molid = -1
        self.name = None
        self.dftb3_energy = float("nan")
        self.dftb3_hof = float("nan")
        self.atomtypes = []
        self.nuclear_charges = []
        self.coordinates = []
        self.active_atoms = []
        self.unit_cell = None
        self.properties = []
        self.properties2 = []

    def _packed(self):
        z = np.asarray(self.nuclear_charges, dtype=np.float64).reshape(-1)
        r = np.asarray(self.coordinates, dtype=np.float64).reshape(-1, 3)
        if len(z) != len(r):
            # frepresentations.f90:45-49
            raise ValueError("ERROR: Coulomb matrix generation: %d coordinates, but %d atom_types!"
                             % (len(r), len(z)))
        return z, r, np.array([0, len(z)], dtype=np.int32)

    def generate_coulomb_matrix(self, size=23):
        """fml/fml.py:64-66 -> sorted CM, packed lower triangle (size*(size+1)/2,)."""
        z, r, off = self._packed()
        self.coulomb_matrix = generate_coulomb_matrices(z, r, off, size=size)[0]

    def generate_unsorted_coulomb_matrix(self, size=23):
        """fml/fml.py:68-70 -> CM in the input atom order, packed lower triangle."""
        z, r, off = self._packed()
        self.unsorted_coulomb_matrix = generate_unsorted_coulomb_matrices(z, r, off, size=size)[0]

    def generate_local_coulomb_matrix(self, calc="all", size=23):
        """fml/fml.py:72-74 -> (natoms, size*(size+1)/2), one row per central atom.

        ``calc`` is accepted and ignored, as in the reference.
        """
        z, r, off = self._packed()
        self.local_coulomb_matrix = generate_local_coulomb_matrices(z, r, off, size=size,
                                                                    kind="local")

    def generate_atomic_coulomb_matrix(self, calc="all", size=23):
        """fml/fml.py:76-78 -> (natoms, size*(size+1)/2), atoms by distance to the centre."""
        z, r, off = self._packed()
        self.atomic_coulomb_matrix = generate_local_coulomb_matrices(z, r, off, size=size,
                                                                     kind="atomic")

    def generate_arad_descriptor(self, size=23):
        """fml/fml.py:80-86 -> ARAD descriptor (size, 5, size), cut 5.0 (fml/arad.py:36)."""
        z, r, off = self._packed()
        self.arad_descriptor = generate_arad_descriptors(z, r, off, size=size, cut=5.0)[0]
        assert (self.arad_descriptor).shape[0] == size, "ERROR: Check ARAD descriptor size!"
        assert (self.arad_descriptor).shape[2] == size, "ERROR: Check ARAD descriptor size!"

    def read_xyz(self, filename):
        """fml/fml.py:109-132: natoms from line 1, atoms from line 3 on."""
        with open(filename, "r") as f:
            lines = f.readlines()
        self.natoms = int(lines[0])
        for line in lines[2:]:
            tokens = line.split()
            if len(tokens) < 4:
                break
            self.atomtypes.append(tokens[0])
            self.nuclear_charges.append(NUCLEAR_CHARGE[tokens[0]])
            self.coordinates.append(np.array([float(tokens[1]), float(tokens[2]),
                                              float(tokens[3])]))
        self.coordinates = np.array(self.coordinates)
