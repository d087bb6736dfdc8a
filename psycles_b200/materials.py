"""Shader graphs, SurfacePrograms and the incremental material library.

Host mirror of the reference's material contract for the in-scope node set:
closures diffuse (Lambert / Oren-Nayar by roughness), glossy (GGX / Beckmann
microfacet reflection), glass and refraction (dielectric microfacet
transmission), emission, transparent, add and mix, fed by constants, float math, conversions, mixes, colour blends
and separate / combine RGB:

  * ShaderGraph / node types       include/psycles/contract/shader_graph.h,
                                   include/psycles/compiler/core_nodes.h:8-101
                                   (type names and socket names and defaults
                                   of src/compiler/core_nodes.cpp)
  * compile_surface_program        src/compiler/surface_program.cpp:381
    -> SurfaceProgram (a topologically ordered value stream + closure tree)
       + SurfaceParameterBlock
  * structure_signature /          src/contract/shader_graph.cpp (graph
    parameter_signature            signatures: structure without socket
                                   literals, literals alone)
  * MaterialLibrary.update         src/compiler/material_library.cpp:25-146:
    same structure signature -> parameters_rebound (program object reused),
    otherwise program_recompiled; a failing update keeps the old revision.

A SurfaceProgram here is exactly what the C ABI consumes (psy_material_desc):
closure instructions whose inputs are either slots of the parameter block
owned by the closure node (unlinked sockets) or value ids of the stream
(linked sockets, PSY_INPUT_VALUE), and value instructions whose
`parameter` operations read slots owned by value nodes.
"""

from __future__ import annotations

import dataclasses
import enum
import hashlib
from typing import Any, Iterable

import numpy as np

from . import _abi


class NodeType(str, enum.Enum):
    # closures (core_nodes.h:79-91)
    DIFFUSE = "psycles.closure.diffuse"
    EMISSION = "psycles.closure.emission"
    TRANSPARENT = "psycles.closure.transparent"
    GLOSSY = "psycles.closure.glossy"
    GLASS = "psycles.closure.glass"
    REFRACTION = "psycles.closure.refraction"
    ADD = "psycles.closure.add"
    MIX = "psycles.closure.mix"
    # values
    CONSTANT_FLOAT = "psycles.constant.float"
    CONSTANT_COLOR = "psycles.constant.color"
    MATH_ADD = "psycles.math.add"
    MATH_SUBTRACT = "psycles.math.subtract"
    MATH_MULTIPLY = "psycles.math.multiply"
    MATH_DIVIDE = "psycles.math.divide"
    MATH_MINIMUM = "psycles.math.minimum"
    MATH_MAXIMUM = "psycles.math.maximum"
    MATH_POWER = "psycles.math.power"
    MATH_ABSOLUTE = "psycles.math.absolute"
    MATH_CLAMP = "psycles.math.clamp"
    CLAMP_RANGE = "psycles.math.clamp_range"
    SCALAR_TO_COLOR = "psycles.convert.scalar_to_color"
    SCALAR_TO_BOOLEAN = "psycles.convert.scalar_to_boolean"
    COLOR_TO_SCALAR = "psycles.convert.color_to_scalar"
    VECTOR_TO_SCALAR = "psycles.convert.vector_to_scalar"
    MIX_FLOAT = "psycles.value.mix_float"
    MIX_VECTOR = "psycles.value.mix_vector"
    MIX_COLOR = "psycles.color.mix"
    MULTIPLY_COLOR = "psycles.color.multiply"
    INVERT_COLOR = "psycles.color.invert"
    SEPARATE_COLOR = "psycles.color.separate"
    COMBINE_COLOR = "psycles.color.combine"


CLOSURE_TYPES = (NodeType.DIFFUSE, NodeType.EMISSION, NodeType.TRANSPARENT, NodeType.GLOSSY, NodeType.GLASS,
                 NodeType.REFRACTION, NodeType.ADD, NodeType.MIX)
GLOSSY_DISTRIBUTIONS = {"GGX": _abi.GLOSSY_GGX, "BECKMANN": _abi.GLOSSY_BECKMANN}
# the Glossy BSDF also takes MULTI_GGX (GGX with Cycles' tabulated energy
# preservation; the scene carries the GGX albedo tables)
GLOSSY_ONLY_DISTRIBUTIONS = {**GLOSSY_DISTRIBUTIONS, "MULTI_GGX": _abi.GLOSSY_MULTI_GGX}

F, C = "float", "color"  # socket kinds: scalar and vector values

# Input sockets (name, kind, default) and outputs (name, kind) per value
# node, as src/compiler/core_nodes.cpp registers them.
_SCHEMA: dict[NodeType, tuple[list, list]] = {
    NodeType.DIFFUSE: ([("Color", C, (0.8, 0.8, 0.8)), ("Roughness", F, 0.0)], []),
    NodeType.EMISSION: ([("Color", C, (1.0, 1.0, 1.0)), ("Strength", F, 1.0)], []),
    NodeType.TRANSPARENT: ([("Color", C, (1.0, 1.0, 1.0))], []),
    NodeType.GLOSSY: ([("Color", C, (0.8, 0.8, 0.8)), ("Roughness", F, 0.2)], []),
    NodeType.GLASS: ([("Color", C, (1.0, 1.0, 1.0)), ("Roughness", F, 0.0), ("IOR", F, 1.5)], []),
    NodeType.REFRACTION: ([("Color", C, (1.0, 1.0, 1.0)), ("Roughness", F, 0.0), ("IOR", F, 1.5)], []),
    NodeType.ADD: ([], []),
    NodeType.MIX: ([("Factor", F, 0.5)], []),
    NodeType.CONSTANT_FLOAT: ([("Value", F, 0.0)], [("Value", F)]),
    NodeType.CONSTANT_COLOR: ([("Color", C, (0.0, 0.0, 0.0))], [("Color", C)]),
    **{t: ([("A", F, 0.0), ("B", F, 0.0)], [("Value", F)])
       for t in (NodeType.MATH_ADD, NodeType.MATH_SUBTRACT, NodeType.MATH_MULTIPLY, NodeType.MATH_DIVIDE,
                 NodeType.MATH_MINIMUM, NodeType.MATH_MAXIMUM, NodeType.MATH_POWER)},
    NodeType.MATH_ABSOLUTE: ([("Value", F, 0.0)], [("Value", F)]),
    NodeType.MATH_CLAMP: ([("Value", F, 0.0)], [("Value", F)]),
    NodeType.CLAMP_RANGE: ([("Value", F, 1.0), ("Min", F, 0.0), ("Max", F, 1.0)], [("Result", F)]),
    NodeType.SCALAR_TO_COLOR: ([("Value", F, 0.0)], [("Color", C)]),
    NodeType.SCALAR_TO_BOOLEAN: ([("Value", F, 0.0)], [("Boolean", F)]),
    NodeType.COLOR_TO_SCALAR: ([("Color", C, (0.0, 0.0, 0.0))], [("Value", F)]),
    NodeType.VECTOR_TO_SCALAR: ([("Vector", C, (0.0, 0.0, 0.0))], [("Value", F)]),
    NodeType.MIX_FLOAT: ([("Factor", F, 0.5), ("A", F, 0.0), ("B", F, 0.0)], [("Value", F)]),
    NodeType.MIX_VECTOR: ([("Factor", F, 0.5), ("A", C, (0.0, 0.0, 0.0)), ("B", C, (0.0, 0.0, 0.0))],
                          [("Vector", C)]),
    NodeType.MIX_COLOR: ([("Factor", F, 0.5), ("A", C, (0.0, 0.0, 0.0)), ("B", C, (1.0, 1.0, 1.0))], [("Color", C)]),
    NodeType.MULTIPLY_COLOR: ([("A", C, (0.0, 0.0, 0.0)), ("B", C, (1.0, 1.0, 1.0)), ("Factor", F, 1.0)],
                              [("Color", C)]),
    NodeType.INVERT_COLOR: ([("Factor", F, 1.0), ("Color", C, (0.8, 0.8, 0.8))], [("Color", C)]),
    NodeType.SEPARATE_COLOR: ([("Color", C, (0.0, 0.0, 0.0))], [("R", F), ("G", F), ("B", F)]),
    NodeType.COMBINE_COLOR: ([("R", F, 0.0), ("G", F, 0.0), ("B", F, 0.0)], [("Color", C)]),
}

_BINARY = {NodeType.MATH_ADD: _abi.VALUE_ADD, NodeType.MATH_SUBTRACT: _abi.VALUE_SUBTRACT,
           NodeType.MATH_MULTIPLY: _abi.VALUE_MULTIPLY, NodeType.MATH_DIVIDE: _abi.VALUE_DIVIDE,
           NodeType.MATH_MINIMUM: _abi.VALUE_MINIMUM, NodeType.MATH_MAXIMUM: _abi.VALUE_MAXIMUM,
           NodeType.MATH_POWER: _abi.VALUE_POWER}
_BLEND = {"MIX": _abi.BLEND_MIX, "DARKEN": _abi.BLEND_DARKEN, "MULTIPLY": _abi.BLEND_MULTIPLY,
          "LIGHTEN": _abi.BLEND_LIGHTEN, "SCREEN": _abi.BLEND_SCREEN, "ADD": _abi.BLEND_ADD,
          "DIFFERENCE": _abi.BLEND_DIFFERENCE, "SUBTRACT": _abi.BLEND_SUBTRACT}


@dataclasses.dataclass(frozen=True)
class Link:
    """A link from output `socket` of value node `node`."""
    node: int
    socket: str


@dataclasses.dataclass
class Node:
    type: NodeType
    sockets: dict[str, Any] = dataclasses.field(default_factory=dict)  # literal or Link
    inputs: tuple[int, ...] = ()                                       # closure children (add / mix)
    props: dict[str, Any] = dataclasses.field(default_factory=dict)    # static properties


class ShaderGraphError(ValueError):
    """A graph that fails validation (validate_shader_graph, src/contract/shader_graph.cpp:319)."""


def _literal(kind: str, value) -> Any:
    if kind == C:
        t = tuple(float(v) for v in value)
        if len(t) != 3:
            raise ShaderGraphError("a colour literal has three components")
        return t
    return float(value)


class ShaderGraph:
    """A shader DAG.  Node ids are indices in topological order; `output`
    names the surface root (a closure node)."""

    def __init__(self) -> None:
        self.nodes: list[Node] = []
        self.output: int | None = None

    def _add(self, node: Node) -> int:
        self.nodes.append(node)
        return len(self.nodes) - 1

    def _node(self, type_: NodeType, props=None, **sockets) -> int:
        names = {n: (k, d) for n, k, d in _SCHEMA[type_][0]}
        values = {}
        for name, value in sockets.items():
            if name not in names:
                raise ShaderGraphError(f"{type_.value} has no input {name}")
            values[name] = value if isinstance(value, Link) else _literal(names[name][0], value)
        for name, (kind, default) in names.items():
            values.setdefault(name, _literal(kind, default))
        return self._add(Node(type_, values, (), dict(props or {})))

    def _out(self, node: int, socket: str | None = None) -> Link:
        outputs = _SCHEMA[self.nodes[node].type][1]
        return Link(node, socket or outputs[0][0])

    # closures
    def diffuse_bsdf(self, color, roughness=0.0) -> int:
        return self._node(NodeType.DIFFUSE, Color=color, Roughness=roughness)

    def glossy_bsdf(self, color, roughness=0.2, distribution: str = "GGX") -> int:
        """Glossy BSDF (core_nodes.cpp:980-990): GGX, Beckmann or MULTI_GGX
        microfacet reflection; the Distribution property is structural."""
        if distribution not in GLOSSY_ONLY_DISTRIBUTIONS:
            raise ShaderGraphError(f"glossy distribution {distribution!r} outside GGX, BECKMANN and MULTI_GGX")
        return self._node(NodeType.GLOSSY, {"Distribution": distribution}, Color=color, Roughness=roughness)

    def glass_bsdf(self, color=(1.0, 1.0, 1.0), roughness=0.0, ior=1.5, distribution: str = "GGX") -> int:
        """Glass BSDF (core_nodes.cpp:992-1004): dielectric microfacet
        reflection and transmission with the Fresnel split; a material may
        hold no other BSDF closure beside it (its selection weight among
        others reads Cycles' tabulated Fresnel albedo)."""
        if distribution not in GLOSSY_DISTRIBUTIONS:
            raise ShaderGraphError(f"glass distribution {distribution!r} outside GGX and BECKMANN")
        return self._node(NodeType.GLASS, {"Distribution": distribution}, Color=color, Roughness=roughness, IOR=ior)

    def refraction_bsdf(self, color=(1.0, 1.0, 1.0), roughness=0.0, ior=1.5, distribution: str = "GGX") -> int:
        """Refraction BSDF (core_nodes.cpp:1006-1019): microfacet
        transmission only."""
        if distribution not in GLOSSY_DISTRIBUTIONS:
            raise ShaderGraphError(f"refraction distribution {distribution!r} outside GGX and BECKMANN")
        return self._node(NodeType.REFRACTION, {"Distribution": distribution}, Color=color, Roughness=roughness, IOR=ior)

    def emission(self, color, strength=1.0) -> int:
        return self._node(NodeType.EMISSION, Color=color, Strength=strength)

    def transparent_bsdf(self, color) -> int:
        return self._node(NodeType.TRANSPARENT, Color=color)

    def add_shader(self, a: int, b: int) -> int:
        return self._add(Node(NodeType.ADD, {}, (a, b)))

    def mix_shader(self, factor, a: int, b: int) -> int:
        node = self._node(NodeType.MIX, Factor=factor)
        self.nodes[node].inputs = (a, b)
        return node

    # values: each returns a Link to the node's (first) output
    def value(self, v) -> Link:
        return self._out(self._node(NodeType.CONSTANT_FLOAT, Value=v))

    def rgb(self, c) -> Link:
        return self._out(self._node(NodeType.CONSTANT_COLOR, Color=c))

    def math(self, op: str, a, b=0.0) -> Link:
        t = NodeType("psycles.math." + op)
        if t in _BINARY:
            return self._out(self._node(t, A=a, B=b))
        return self._out(self._node(t, Value=a))

    def clamp_range(self, value, lo, hi, mode: str = "MINMAX") -> Link:
        return self._out(self._node(NodeType.CLAMP_RANGE, {"Mode": mode}, Value=value, Min=lo, Max=hi))

    def convert(self, kind: str, value) -> Link:
        t = NodeType("psycles.convert." + kind)
        name = _SCHEMA[t][0][0][0]
        return self._out(self._node(t, **{name: value}))

    def mix_float(self, factor, a, b, clamp: bool = True) -> Link:
        return self._out(self._node(NodeType.MIX_FLOAT, {"ClampFactor": clamp}, Factor=factor, A=a, B=b))

    def mix_vector(self, factor, a, b, clamp: bool = True) -> Link:
        return self._out(self._node(NodeType.MIX_VECTOR, {"ClampFactor": clamp}, Factor=factor, A=a, B=b))

    def mix_color(self, factor, a, b, blend: str = "MIX", clamp: bool = True) -> Link:
        return self._out(self._node(NodeType.MIX_COLOR, {"BlendMode": blend, "ClampFactor": clamp},
                                    Factor=factor, A=a, B=b))

    def multiply_color(self, a, b, factor=1.0) -> Link:
        return self._out(self._node(NodeType.MULTIPLY_COLOR, A=a, B=b, Factor=factor))

    def invert_color(self, factor, color) -> Link:
        return self._out(self._node(NodeType.INVERT_COLOR, Factor=factor, Color=color))

    def separate_color(self, color) -> tuple[Link, Link, Link]:
        node = self._node(NodeType.SEPARATE_COLOR, {"Mode": "RGB"}, Color=color)
        return Link(node, "R"), Link(node, "G"), Link(node, "B")

    def combine_color(self, r, g, b) -> Link:
        return self._out(self._node(NodeType.COMBINE_COLOR, {"Mode": "RGB"}, R=r, G=g, B=b))

    def set_output(self, node: int) -> "ShaderGraph":
        self.output = node
        return self

    def validate(self) -> None:
        if self.output is None or not 0 <= self.output < len(self.nodes):
            raise ShaderGraphError("graph has no surface output")
        if self.nodes[self.output].type not in CLOSURE_TYPES:
            raise ShaderGraphError("the surface output is not a closure")
        for i, n in enumerate(self.nodes):
            for j in n.inputs:
                if not 0 <= j < i:
                    raise ShaderGraphError(f"node {i} closure input {j} is not an earlier node")
                if self.nodes[j].type not in CLOSURE_TYPES:
                    raise ShaderGraphError(f"node {i} closure input {j} is not a closure")
            for name, v in n.sockets.items():
                if isinstance(v, Link):
                    if not 0 <= v.node < len(self.nodes) or self.nodes[v.node].type in CLOSURE_TYPES:
                        raise ShaderGraphError(f"node {i} input {name} links a node that is not a value node")
                    if v.socket not in {o for o, _ in _SCHEMA[self.nodes[v.node].type][1]}:
                        raise ShaderGraphError(f"node {i} input {name} links a missing output {v.socket}")
            if n.type in (NodeType.ADD, NodeType.MIX) and len(n.inputs) != 2:
                raise ShaderGraphError(f"node {i} needs two closure inputs")
            if n.type == NodeType.MIX_COLOR:
                if n.props.get("BlendMode", "MIX") not in _BLEND:
                    raise ShaderGraphError(f"blend mode {n.props.get('BlendMode')} is not supported")
                if n.props.get("ClampResult", False):
                    raise ShaderGraphError("mix colour ClampResult is not supported")
            if n.type in (NodeType.SEPARATE_COLOR, NodeType.COMBINE_COLOR) and n.props.get("Mode", "RGB") != "RGB":
                raise ShaderGraphError("separate / combine colour only in RGB mode")
        # value links form a DAG (values are lowered operands first)
        state = [0] * len(self.nodes)

        def visit(i: int) -> None:
            if state[i] == 2:
                return
            if state[i] == 1:
                raise ShaderGraphError(f"value links form a cycle through node {i}")
            state[i] = 1
            for v in self.nodes[i].sockets.values():
                if isinstance(v, Link):
                    visit(v.node)
            state[i] = 2

        for i in range(len(self.nodes)):
            visit(i)

    def structure_signature(self) -> str:
        """Hash of node types, links and static properties, without socket literals."""
        h = hashlib.sha256()
        for n in self.nodes:
            links = sorted((k, v.node, v.socket) for k, v in n.sockets.items() if isinstance(v, Link))
            h.update(f"{n.type.value}:{n.inputs}:{links}:{sorted(n.props.items())};".encode())
        h.update(f"out:{self.output}".encode())
        return h.hexdigest()[:16]

    def parameter_signature(self) -> str:
        h = hashlib.sha256()
        for n in self.nodes:
            lits = sorted((k, v) for k, v in n.sockets.items() if not isinstance(v, Link))
            h.update(f"{lits};".encode())
        return h.hexdigest()[:16]


@dataclasses.dataclass
class SurfaceParameterBlock:
    scalars: np.ndarray  # float32[scalar_count]
    vectors: np.ndarray  # float32[vector_count, 3]


@dataclasses.dataclass
class SurfaceProgram:
    closures: np.ndarray  # ClosureInstruction rows (6 x uint32)
    values: np.ndarray    # ValueInstruction rows (8 x uint32)
    root: int
    scalar_count: int
    vector_count: int
    structure_signature: str
    has_emission: bool
    has_transparent: bool


class _Lowering:
    """One pass over a validated graph: value nodes become value
    instructions on first use (operands first), literals of value nodes
    become `parameter` instructions, literals of closure nodes stay direct
    slots of the block."""

    def __init__(self, graph: ShaderGraph):
        self.g = graph
        self.scalars: list[float] = []
        self.vectors: list[tuple] = []
        self.values: list[tuple] = []
        self.memo: dict[tuple[int, str], int] = {}

    def emit(self, op, kind, a=0, b=0, c=0, u0=0, u1=0, parameter=0) -> int:
        t = _abi.VALUE_TYPE_VECTOR if kind == C else _abi.VALUE_TYPE_SCALAR
        self.values.append((op, t, parameter, a, b, c, u0, u1))
        return len(self.values) - 1

    def kind_of(self, vid: int) -> str:
        return C if self.values[vid][1] == _abi.VALUE_TYPE_VECTOR else F

    def slot(self, kind: str, literal) -> int:
        if kind == C:
            self.vectors.append(literal)
            return len(self.vectors) - 1
        self.scalars.append(literal)
        return len(self.scalars) - 1

    def convert(self, vid: int, kind: str) -> int:
        """Implicit socket conversion of a link (float <-> colour)."""
        have = self.kind_of(vid)
        if have == kind:
            return vid
        if kind == C:
            return self.emit(_abi.VALUE_SCALAR_TO_COLOR, C, a=vid)
        return self.emit(_abi.VALUE_COLOR_TO_SCALAR, F, a=vid)

    def value_input(self, node: Node, name: str) -> int:
        """Value id of a value node's input socket."""
        kind = next(k for n, k, _ in _SCHEMA[node.type][0] if n == name)
        v = node.sockets[name]
        if isinstance(v, Link):
            return self.convert(self.output(v), kind)
        return self.emit(_abi.VALUE_PARAMETER, kind, parameter=self.slot(kind, v))

    def closure_input(self, node: Node, name: str) -> int:
        """Closure input encoding: a direct slot, or PSY_INPUT_VALUE | id."""
        kind = next(k for n, k, _ in _SCHEMA[node.type][0] if n == name)
        v = node.sockets[name]
        if isinstance(v, Link):
            return _abi.INPUT_VALUE | self.convert(self.output(v), kind)
        return self.slot(kind, v)

    def output(self, link: Link) -> int:
        key = (link.node, link.socket)
        if key in self.memo:
            return self.memo[key]
        n = self.g.nodes[link.node]
        t = n.type
        vi = lambda name: self.value_input(n, name)
        if t in (NodeType.CONSTANT_FLOAT, NodeType.CONSTANT_COLOR):
            out = vi(_SCHEMA[t][0][0][0])
        elif t in _BINARY:
            a, b = vi("A"), vi("B")
            out = self.emit(_BINARY[t], F, a=a, b=b)
        elif t == NodeType.MATH_ABSOLUTE:
            out = self.emit(_abi.VALUE_ABSOLUTE, F, a=vi("Value"))
        elif t == NodeType.MATH_CLAMP:
            out = self.emit(_abi.VALUE_CLAMP01, F, a=vi("Value"))
        elif t == NodeType.CLAMP_RANGE:
            a, b, c = vi("Value"), vi("Min"), vi("Max")
            out = self.emit(_abi.VALUE_CLAMP_RANGE, F, a=a, b=b, c=c, u0=1 if n.props.get("Mode") == "RANGE" else 0)
        elif t == NodeType.SCALAR_TO_COLOR:
            out = self.emit(_abi.VALUE_SCALAR_TO_COLOR, C, a=vi("Value"))
        elif t == NodeType.SCALAR_TO_BOOLEAN:
            out = self.emit(_abi.VALUE_SCALAR_TO_BOOLEAN, F, a=vi("Value"))
        elif t == NodeType.COLOR_TO_SCALAR:
            out = self.emit(_abi.VALUE_COLOR_TO_SCALAR, F, a=vi("Color"))
        elif t == NodeType.VECTOR_TO_SCALAR:
            out = self.emit(_abi.VALUE_VECTOR_TO_SCALAR, F, a=vi("Vector"))
        elif t == NodeType.MIX_FLOAT:
            f, a, b = vi("Factor"), vi("A"), vi("B")
            out = self.emit(_abi.VALUE_MIX_FLOAT, F, a=a, b=b, c=f, u0=int(bool(n.props.get("ClampFactor", True))))
        elif t == NodeType.MIX_VECTOR:
            f, a, b = vi("Factor"), vi("A"), vi("B")
            out = self.emit(_abi.VALUE_MIX_VECTOR, C, a=a, b=b, c=f, u0=0,
                            u1=int(bool(n.props.get("ClampFactor", True))))
        elif t == NodeType.MIX_COLOR:
            f, a, b = vi("Factor"), vi("A"), vi("B")
            out = self.emit(_abi.VALUE_MIX, C, a=a, b=b, c=f, u0=_BLEND[n.props.get("BlendMode", "MIX")],
                            u1=int(bool(n.props.get("ClampFactor", True))))
        elif t == NodeType.MULTIPLY_COLOR:
            a, b, f = vi("A"), vi("B"), vi("Factor")
            out = self.emit(_abi.VALUE_MULTIPLY_COLOR, C, a=a, b=b, c=f)
        elif t == NodeType.INVERT_COLOR:
            f, col = vi("Factor"), vi("Color")
            out = self.emit(_abi.VALUE_INVERT, C, a=col, b=f)
        elif t == NodeType.SEPARATE_COLOR:
            col = vi("Color")
            op = {"R": _abi.VALUE_SEPARATE_R, "G": _abi.VALUE_SEPARATE_G, "B": _abi.VALUE_SEPARATE_B}[link.socket]
            out = self.emit(op, F, a=col)
        elif t == NodeType.COMBINE_COLOR:
            r, g, b = vi("R"), vi("G"), vi("B")
            out = self.emit(_abi.VALUE_COMBINE_COLOR, C, a=r, b=g, c=b)
        else:
            raise ShaderGraphError(f"{t.value} has no value output")
        self.memo[key] = out
        return out


def compile_surface_program(graph: ShaderGraph) -> tuple[SurfaceProgram, SurfaceParameterBlock]:
    """Lowers a validated graph to a value stream + closure tree plus its
    parameter block.  Closure instruction k is node k's closure (value nodes
    hold null closures, which the tree never reaches)."""
    graph.validate()
    low = _Lowering(graph)
    none = _abi.INPUT_NONE
    code: list[tuple] = []
    for n in graph.nodes:
        if n.type == NodeType.DIFFUSE:
            code.append((_abi.CLOSURE_DIFFUSE, 0, 0, low.closure_input(n, "Color"), none,
                         low.closure_input(n, "Roughness")))
        elif n.type == NodeType.TRANSPARENT:
            code.append((_abi.CLOSURE_TRANSPARENT, 0, 0, low.closure_input(n, "Color"), none, none))
        elif n.type == NodeType.GLOSSY:
            code.append((_abi.CLOSURE_GLOSSY, GLOSSY_ONLY_DISTRIBUTIONS[n.props.get("Distribution", "GGX")], 0,
                         low.closure_input(n, "Color"), none, low.closure_input(n, "Roughness")))
        elif n.type in (NodeType.GLASS, NodeType.REFRACTION):
            op = _abi.CLOSURE_GLASS if n.type == NodeType.GLASS else _abi.CLOSURE_REFRACTION
            code.append((op, GLOSSY_DISTRIBUTIONS[n.props.get("Distribution", "GGX")], 0,
                         low.closure_input(n, "Color"), low.closure_input(n, "IOR"), low.closure_input(n, "Roughness")))
        elif n.type == NodeType.EMISSION:
            code.append((_abi.CLOSURE_EMISSION, 0, 0, low.closure_input(n, "Color"), low.closure_input(n, "Strength"),
                         none))
        elif n.type == NodeType.ADD:
            code.append((_abi.CLOSURE_ADD, n.inputs[0], n.inputs[1], none, none, none))
        elif n.type == NodeType.MIX:
            code.append((_abi.CLOSURE_MIX, n.inputs[0], n.inputs[1], none, low.closure_input(n, "Factor"), none))
        else:
            code.append((_abi.CLOSURE_NULL, 0, 0, none, none, none))
    program = SurfaceProgram(
        closures=np.ascontiguousarray(np.array(code, dtype=np.uint32).reshape(-1, 6)),
        values=np.ascontiguousarray(np.array(low.values, dtype=np.uint32).reshape(-1, 8)),
        root=int(graph.output), scalar_count=len(low.scalars), vector_count=len(low.vectors),
        structure_signature=graph.structure_signature(),
        has_emission=any(n.type == NodeType.EMISSION for n in graph.nodes),
        has_transparent=any(n.type == NodeType.TRANSPARENT for n in graph.nodes))
    block = SurfaceParameterBlock(
        scalars=np.array(low.scalars, dtype=np.float32).reshape(-1),
        vectors=np.array(low.vectors, dtype=np.float32).reshape(-1, 3))
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
    use_bump_map_correction: bool = True


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
                    staged[name] = CompiledMaterial(graph, old.program, block, old.emission_sampling,
                                                    old.use_bump_map_correction)
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


def diffuse_material(color, roughness: float = 0.0) -> ShaderGraph:
    g = ShaderGraph()
    return g.set_output(g.diffuse_bsdf(color, roughness))


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


def glass_material(color=(1.0, 1.0, 1.0), roughness: float = 0.0, ior: float = 1.5,
                   distribution: str = "GGX") -> ShaderGraph:
    g = ShaderGraph()
    return g.set_output(g.glass_bsdf(color, roughness, ior, distribution))


def glossy_material(color, roughness: float = 0.2, distribution: str = "GGX") -> ShaderGraph:
    g = ShaderGraph()
    return g.set_output(g.glossy_bsdf(color, roughness, distribution))


def glossy_mixture_material(rng: np.random.Generator) -> ShaderGraph:
    """A random mixture with glossy lobes: diffuse + glossy (mix or add),
    glossy over a transparent closure, or glossy with a roughness linked to
    a Value node; GGX or Beckmann, roughness 0 (a mirror: singular) to 0.8."""
    g = ShaderGraph()
    dist = "BECKMANN" if rng.random() < 0.35 else "GGX"
    rough = 0.0 if rng.random() < 0.2 else float(rng.uniform(0.05, 0.8))
    color = tuple(float(v) for v in rng.uniform(0.3, 0.95, 3))
    kind = int(rng.integers(0, 4))
    if kind == 0:
        gl = g.glossy_bsdf(color, rough, dist)
        d = g.diffuse_bsdf(tuple(float(v) for v in rng.uniform(0.1, 0.8, 3)), float(rng.uniform(0.0, 0.6)))
        return g.set_output(g.mix_shader(float(rng.uniform(0.1, 0.9)), d, gl))
    if kind == 1:
        gl = g.glossy_bsdf(color, rough, dist)
        d = g.diffuse_bsdf(tuple(float(v) for v in rng.uniform(0.1, 0.5, 3)))
        return g.set_output(g.add_shader(d, gl))
    if kind == 2:
        gl = g.glossy_bsdf(color, rough, dist)
        t = g.transparent_bsdf(tuple(float(v) for v in rng.uniform(0.4, 0.9, 3)))
        return g.set_output(g.mix_shader(float(rng.uniform(0.2, 0.8)), gl, t))
    r = g.math("multiply", g.value(float(rng.uniform(0.1, 0.9))), float(rng.uniform(0.3, 1.0)))
    return g.set_output(g.glossy_bsdf(color, r, dist))


def value_graph_material(rng: np.random.Generator) -> ShaderGraph:
    """A random graph whose closure inputs are linked to value nodes: an RGB
    node through a colour blend into a rough diffuse colour, a Value node
    through float math into a mix factor and an emission strength, separate
    / combine RGB and the float <-> colour conversions."""
    g = ShaderGraph()
    base = g.rgb(tuple(float(v) for v in rng.uniform(0.1, 0.9, 3)))
    tint = g.rgb(tuple(float(v) for v in rng.uniform(0.1, 0.9, 3)))
    blend = ["MIX", "MULTIPLY", "SCREEN", "DARKEN", "LIGHTEN", "ADD", "SUBTRACT", "DIFFERENCE"][int(rng.integers(0, 8))]
    color = g.mix_color(float(rng.uniform(0.0, 1.0)), base, tint, blend=blend)
    r, gg, b = g.separate_color(color)
    swizzled = g.combine_color(gg, b, r)
    fac = g.math("clamp", g.math("multiply", g.value(float(rng.uniform(0.2, 2.0))), float(rng.uniform(0.1, 0.9))))
    rough = g.math("power", g.value(float(rng.uniform(0.1, 0.9))), float(rng.uniform(0.5, 2.0)))
    d1 = g.diffuse_bsdf(g.invert_color(float(rng.uniform(0.0, 0.5)), swizzled), rough)
    d2 = g.diffuse_bsdf(g.multiply_color(color, g.convert("scalar_to_color", fac), 0.8),
                        float(rng.uniform(0.0, 1.0)))
    mixed = g.mix_shader(fac, d1, d2)
    if rng.random() < 0.3:
        strength = g.mix_float(float(rng.uniform(0.0, 1.0)), 0.5, g.convert("color_to_scalar", tint))
        mixed = g.add_shader(mixed, g.emission(g.mix_vector(0.5, base, tint), strength))
    if rng.random() < 0.3:
        mixed = g.mix_shader(g.clamp_range(g.value(float(rng.uniform(-0.5, 1.5))), 0.1, 0.6),
                             mixed, g.transparent_bsdf((0.9, 0.9, 0.9)))
    return g.set_output(mixed)


def iter_closure_counts(graphs: Iterable[ShaderGraph]) -> list[int]:
    return [sum(1 for n in g.nodes if n.type in (NodeType.DIFFUSE, NodeType.EMISSION, NodeType.TRANSPARENT))
            for g in graphs]
