"""Shader graphs, SurfacePrograms and the incremental material library.

Host mirror of the reference's material contract for the in-scope closure
set (diffuse, emission, transparent, add, mix with uniform colour and scalar
inputs):

  * ShaderGraph / node types       include/psycles/contract/shader_graph.h,
                                   include/psycles/compiler/core_nodes.h:79-91
  * compile_surface_program        src/compiler/surface_program.cpp:381
    -> SurfaceProgram (closure instruction tree) + SurfaceParameterBlock
  * structure_signature /          src/contract/shader_graph.cpp (graph
    parameter_signature            signatures: structure without constant
                                   values, values alone)
  * MaterialLibrary.update         src/compiler/material_library.cpp:25-146:
    same structure signature -> parameters_rebound (program object reused),
    otherwise program_recompiled; a failing update keeps the old revision.

A SurfaceProgram here is exactly what the C ABI consumes
(psy_material_desc): closure instructions whose colour / factor inputs name
slots of the parameter block.
"""

from __future__ import annotations

import dataclasses
import enum
import hashlib
from typing import Iterable

import numpy as np

from . import _abi


class NodeType(str, enum.Enum):
    DIFFUSE = "psycles.closure.diffuse"
    EMISSION = "psycles.closure.emission"
    TRANSPARENT = "psycles.closure.transparent"
    ADD = "psycles.closure.add"
    MIX = "psycles.closure.mix"


@dataclasses.dataclass
class Node:
    type: NodeType
    color: tuple[float, float, float] | None = None
    strength: float | None = None
    factor: float | None = None
    inputs: tuple[int, ...] = ()


class ShaderGraphError(ValueError):
    """A graph that fails validation (validate_shader_graph, src/contract/shader_graph.cpp:319)."""


class ShaderGraph:
    """A closure DAG.  Node ids are indices; `output` names the surface root."""

    def __init__(self) -> None:
        self.nodes: list[Node] = []
        self.output: int | None = None

    def _add(self, node: Node) -> int:
        self.nodes.append(node)
        return len(self.nodes) - 1

    def diffuse_bsdf(self, color) -> int:
        return self._add(Node(NodeType.DIFFUSE, color=tuple(float(c) for c in color)))

    def emission(self, color, strength: float) -> int:
        return self._add(Node(NodeType.EMISSION, color=tuple(float(c) for c in color), strength=float(strength)))

    def transparent_bsdf(self, color) -> int:
        return self._add(Node(NodeType.TRANSPARENT, color=tuple(float(c) for c in color)))

    def add_shader(self, a: int, b: int) -> int:
        return self._add(Node(NodeType.ADD, inputs=(a, b)))

    def mix_shader(self, factor: float, a: int, b: int) -> int:
        return self._add(Node(NodeType.MIX, factor=float(factor), inputs=(a, b)))

    def set_output(self, node: int) -> "ShaderGraph":
        self.output = node
        return self

    def validate(self) -> None:
        if self.output is None or not 0 <= self.output < len(self.nodes):
            raise ShaderGraphError("graph has no surface output")
        for i, n in enumerate(self.nodes):
            for j in n.inputs:
                if not 0 <= j < len(self.nodes):
                    raise ShaderGraphError(f"node {i} input {j} out of range")
                if j >= i:
                    raise ShaderGraphError(f"node {i} input {j} is not topologically earlier")
            if n.type in (NodeType.DIFFUSE, NodeType.EMISSION, NodeType.TRANSPARENT) and n.color is None:
                raise ShaderGraphError(f"node {i} lacks a colour")

    def structure_signature(self) -> str:
        """Hash of node types and topology without constant values."""
        h = hashlib.sha256()
        for n in self.nodes:
            h.update(f"{n.type.value}:{n.inputs};".encode())
        h.update(f"out:{self.output}".encode())
        return h.hexdigest()[:16]

    def parameter_signature(self) -> str:
        h = hashlib.sha256()
        for n in self.nodes:
            h.update(f"{n.color}:{n.strength}:{n.factor};".encode())
        return h.hexdigest()[:16]


@dataclasses.dataclass
class SurfaceParameterBlock:
    scalars: np.ndarray  # float32[scalar_count]
    vectors: np.ndarray  # float32[vector_count, 3]


@dataclasses.dataclass
class SurfaceProgram:
    closures: np.ndarray  # structured ClosureInstruction array (5 x uint32 per entry)
    root: int
    scalar_count: int
    vector_count: int
    structure_signature: str
    has_emission: bool
    has_transparent: bool


def compile_surface_program(graph: ShaderGraph) -> tuple[SurfaceProgram, SurfaceParameterBlock]:
    """Lowers a validated graph to a closure tree plus its parameter block."""
    graph.validate()
    scalars: list[float] = []
    vectors: list[tuple[float, float, float]] = []
    code: list[tuple[int, int, int, int, int]] = []
    for n in graph.nodes:
        if n.type == NodeType.DIFFUSE:
            vectors.append(n.color)
            code.append((_abi.CLOSURE_DIFFUSE, 0, 0, len(vectors) - 1, 0))
        elif n.type == NodeType.TRANSPARENT:
            vectors.append(n.color)
            code.append((_abi.CLOSURE_TRANSPARENT, 0, 0, len(vectors) - 1, 0))
        elif n.type == NodeType.EMISSION:
            vectors.append(n.color)
            scalars.append(n.strength)
            code.append((_abi.CLOSURE_EMISSION, 0, 0, len(vectors) - 1, len(scalars) - 1))
        elif n.type == NodeType.ADD:
            code.append((_abi.CLOSURE_ADD, n.inputs[0], n.inputs[1], 0, 0))
        elif n.type == NodeType.MIX:
            scalars.append(n.factor)
            code.append((_abi.CLOSURE_MIX, n.inputs[0], n.inputs[1], 0, len(scalars) - 1))
    arr = np.array(code, dtype=np.uint32).reshape(-1, 5)
    program = SurfaceProgram(
        closures=np.ascontiguousarray(arr), root=int(graph.output), scalar_count=len(scalars),
        vector_count=len(vectors), structure_signature=graph.structure_signature(),
        has_emission=any(n.type == NodeType.EMISSION for n in graph.nodes),
        has_transparent=any(n.type == NodeType.TRANSPARENT for n in graph.nodes))
    block = SurfaceParameterBlock(
        scalars=np.array(scalars, dtype=np.float32).reshape(-1),
        vectors=np.array(vectors, dtype=np.float32).reshape(-1, 3))
    return program, block


def bind_surface_parameters(program: SurfaceProgram, graph: ShaderGraph) -> SurfaceParameterBlock:
    """New parameter block for a graph of the same structure (surface_program.cpp:386)."""
    if graph.structure_signature() != program.structure_signature:
        raise ShaderGraphError("graph structure differs from the compiled program")
    _, block = compile_surface_program(graph)
    return block


class MaterialUpdateKind(str, enum.Enum):
    """compiler::MaterialUpdateKind (include/psycles/compiler/material_library.h:14)."""
    UNCHANGED = "unchanged"
    ADDED = "added"
    PARAMETERS_REBOUND = "parameters_rebound"
    PROGRAM_RECOMPILED = "program_recompiled"
    REMOVED = "removed"


@dataclasses.dataclass
class CompiledMaterial:
    graph: ShaderGraph
    program: SurfaceProgram
    parameters: SurfaceParameterBlock
    emission_sampling: int = _abi.EMISSION_AUTOMATIC


class MaterialLibrary:
    """Incremental, atomic material library keyed by material name."""

    def __init__(self) -> None:
        self.revision = 0
        self.materials: dict[str, CompiledMaterial] = {}

    def update(self, graphs: dict[str, ShaderGraph]) -> dict[str, MaterialUpdateKind]:
        staged: dict[str, CompiledMaterial] = {}
        kinds: dict[str, MaterialUpdateKind] = {}
        for name, graph in graphs.items():
            old = self.materials.get(name)
            if old is not None and old.graph.structure_signature() == graph.structure_signature():
                if old.graph.parameter_signature() == graph.parameter_signature():
                    staged[name] = old
                    kinds[name] = MaterialUpdateKind.UNCHANGED
                else:
                    block = bind_surface_parameters(old.program, graph)  # raises before commit
                    staged[name] = CompiledMaterial(graph, old.program, block, old.emission_sampling)
                    kinds[name] = MaterialUpdateKind.PARAMETERS_REBOUND
            else:
                program, block = compile_surface_program(graph)  # raises before commit
                staged[name] = CompiledMaterial(graph, program, block)
                kinds[name] = MaterialUpdateKind.ADDED if old is None else MaterialUpdateKind.PROGRAM_RECOMPILED
        for name in self.materials:
            if name not in graphs:
                kinds[name] = MaterialUpdateKind.REMOVED
        self.materials = staged
        self.revision += 1
        return kinds


def diffuse_material(color) -> ShaderGraph:
    g = ShaderGraph()
    return g.set_output(g.diffuse_bsdf(color))


def emission_material(color, strength: float) -> ShaderGraph:
    g = ShaderGraph()
    return g.set_output(g.emission(color, strength))


def random_material(rng: np.random.Generator, max_leaves: int = 6, emission_probability: float = 0.1,
                    transparent_probability: float = 0.15) -> ShaderGraph:
    """Random closure graph over diffuse / emission / transparent / add / mix."""
    g = ShaderGraph()
    leaves = int(rng.integers(1, max_leaves + 1))
    ids = []
    for _ in range(leaves):
        u = rng.random()
        color = tuple(float(v) for v in rng.uniform(0.05, 0.9, 3))
        if u < emission_probability:
            ids.append(g.emission(color, float(rng.uniform(0.5, 4.0))))
        elif u < emission_probability + transparent_probability:
            ids.append(g.transparent_bsdf(tuple(float(v) for v in rng.uniform(0.3, 0.95, 3))))
        else:
            ids.append(g.diffuse_bsdf(color))
    while len(ids) > 1:
        a = ids.pop(0)
        b = ids.pop(0)
        if rng.random() < 0.5:
            ids.append(g.mix_shader(float(rng.uniform(0.0, 1.0)), a, b))
        else:
            ids.append(g.add_shader(a, b))
    return g.set_output(ids[0])


def iter_closure_counts(graphs: Iterable[ShaderGraph]) -> list[int]:
    return [sum(1 for n in g.nodes if n.type in (NodeType.DIFFUSE, NodeType.EMISSION, NodeType.TRANSPARENT))
            for g in graphs]
