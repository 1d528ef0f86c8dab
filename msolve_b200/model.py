"""Host-side model for the Hexa8 path: structured block generation, DOF
numbering and nodal loads, mirroring the reference's preprocessor.

- ``Hexa8MeshGenerator.block`` follows Hexa8MeshGenerator.BuildNodes
  (ISAAR.MSolve.SimpleMeshGenerator/Hexa8MeshGenerator.cs:508-568: node IDs x
  fastest, then y, then z) and the element corner order of :1075-1089.
- ``Model.ConnectDataStructures`` numbers free DOFs as Model.EnumerateGlobalDOFs
  (ISAAR.MSolve.PreProcessor/Model.cs:165-215): ascending node ID, X, Y, Z,
  constrained -> -1; loads are *assigned* per DOF (Model.AssignNodalLoads
  :227-238), so a caller that wants accumulated loads sums them first.
"""
from __future__ import annotations

import numpy as np

X, Y, Z = 0, 1, 2


class Subdomain:
    """ISolverSubdomain analogue: RHS (Forces), Solution, DOF map."""

    def __init__(self, model):
        self.model = model
        self.ID = 1
        self.Forces = None
        self.Solution = None

    @property
    def RHS(self):
        return self.Forces

    @property
    def TotalDOFs(self):
        return self.model.n_dofs


class Model:
    """Nodes, Hexa8 elements, constraints, nodal loads and material data."""

    def __init__(self, xyz, conn, young=1.0, poisson=0.3, density=1.0):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.constraints = np.zeros((self.xyz.shape[0], 3), dtype=bool)
        self.loads = []  # (node, dof_type, amount)
        self.young = float(young)
        self.poisson = float(poisson)
        self.density = float(density)
        self.E_elem = np.full(self.conn.shape[0], self.young)
        self.dof = None
        self.n_dofs = 0
        self.subdomains = [Subdomain(self)]
        self.structured = None  # (nx, ny, nz, h) when generated as a block

    @property
    def n_nodes(self):
        return self.xyz.shape[0]

    @property
    def n_elems(self):
        return self.conn.shape[0]

    def constrain(self, nodes, dofs=(X, Y, Z)):
        for d in dofs:
            self.constraints[nodes, d] = True

    def add_load(self, node, dof_type, amount):
        self.loads.append((int(node), int(dof_type), float(amount)))

    def ConnectDataStructures(self):
        """EnumerateGlobalDOFs + AssignNodalLoads."""
        dof = np.full((self.n_nodes, 3), -1, dtype=np.int32)
        free = ~self.constraints
        dof[free] = np.arange(int(free.sum()), dtype=np.int32)
        self.dof = dof
        self.n_dofs = int(free.sum())
        f = np.zeros(self.n_dofs)
        for node, d, amount in self.loads:
            k = dof[node, d]
            if k >= 0:
                f[k] = amount  # assignment, as Model.AssignNodalLoads (:236)
        for s in self.subdomains:
            s.Forces = f
        return self

    def element_xyz(self):
        return self.xyz[self.conn].reshape(self.n_elems, 24)

    def dof_of(self, node, dof_type):
        return int(self.dof[node, dof_type])


class Hexa8MeshGenerator:
    """Structured blocks of unit-spaced Hexa8 elements (generator order)."""

    @staticmethod
    def block(nx, ny, nz, h=1.0, young=1.0, poisson=0.3, density=1.0):
        i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
        # node id = i + (nx+1)(j + (ny+1)k): flatten with x fastest
        xyz = np.stack([i.transpose(2, 1, 0).ravel(), j.transpose(2, 1, 0).ravel(), k.transpose(2, 1, 0).ravel()],
                       axis=1).astype(np.float64) * h
        NX, NXY = nx + 1, (nx + 1) * (ny + 1)
        ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        base = (ei + NX * ej + NXY * ek).transpose(2, 1, 0).ravel()
        conn = np.stack([base, base + 1, base + NX + 1, base + NX, base + NXY, base + NXY + 1, base + NXY + NX + 1,
                         base + NXY + NX], axis=1).astype(np.int32)
        m = Model(xyz, conn, young, poisson, density)
        m.structured = (nx, ny, nz, h)
        return m

    @staticmethod
    def clamp_plane(model, axis, value=0.0):
        nodes = np.nonzero(np.isclose(model.xyz[:, axis], value))[0]
        model.constrain(nodes)
        return nodes

    @staticmethod
    def tip_load(model, axis=X, direction=Z, total=-1.0):
        """Total load split equally over the nodes of the face at the maximum of `axis`."""
        face = np.nonzero(np.isclose(model.xyz[:, axis], model.xyz[:, axis].max()))[0]
        for n in face:
            model.add_load(n, direction, total / len(face))
        return face

    @staticmethod
    def top_pressure(model, p=1.0):
        """Uniform pressure p in -z on the top face, consistent bilinear weights
        (p h^2 / 4 per adjacent top-face element: interior 1, edge 1/2, corner 1/4)."""
        nx, ny, nz, h = model.structured
        top = np.nonzero(np.isclose(model.xyz[:, 2], model.xyz[:, 2].max()))[0]
        xs, ys = model.xyz[top, 0] / h, model.xyz[top, 1] / h
        cx = np.where(np.isclose(xs, 0) | np.isclose(xs, nx), 1, 2)
        cy = np.where(np.isclose(ys, 0) | np.isclose(ys, ny), 1, 2)
        for n, a, b in zip(top, cx, cy):
            model.add_load(n, Z, -p * h * h * a * b / 4.0)
        return top


def cantilever_model(nx=10, ny=4, nz=4, young=1.0, poisson=0.3, total=-1.0):
    """Linear-static cantilever: x=0 face clamped, total load in z split over the x=max face."""
    m = Hexa8MeshGenerator.block(nx, ny, nz, 1.0, young, poisson)
    Hexa8MeshGenerator.clamp_plane(m, X, 0.0)
    Hexa8MeshGenerator.tip_load(m, X, Z, total)
    return m.ConnectDataStructures()


def clamped_block_model(n, young=1.0, poisson=0.3, p=1.0, ny=None, nz=None):
    """n^3 block of unit cubes, z=0 face clamped, unit pressure on the top face."""
    m = Hexa8MeshGenerator.block(n, ny or n, nz or n, 1.0, young, poisson)
    Hexa8MeshGenerator.clamp_plane(m, Z, 0.0)
    Hexa8MeshGenerator.top_pressure(m, p)
    return m.ConnectDataStructures()


def tip_dof(model):
    """u_z of the node at the far corner (max x, max y, max z)."""
    xyz = model.xyz
    n = int(np.argmax(xyz[:, 0] + xyz[:, 1] * 1e3 + xyz[:, 2] * 1e6))
    return model.dof_of(n, Z)


class MassAccelerationSinusoidalLoad:
    """Ground acceleration history (MassAccelerationSinusoidalLoad.cs:11-31):
    load[i] = magnitude sin(2 pi / period * timeStep * i) for i < int(timeLength /
    timeStep), else 0; dof 0/1/2 = X/Y/Z (the DOFType it acts on)."""

    def __init__(self, period, time_step, time_length, magnitude, dof=0):
        self.period, self.time_step, self.time_length, self.magnitude = period, time_step, time_length, magnitude
        self.dof = dof
        self.time_steps = int(time_length / time_step)

    def __getitem__(self, step):
        import math
        return self.magnitude * math.sin(2 * math.pi / self.period * self.time_step * step) \
            if step < self.time_steps else 0.0
