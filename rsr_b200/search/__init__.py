"""Genetic search over the engine: the reference's island model with every
evaluation phase batched across islands (see engine.py)."""
from .engine import (BASIC, LINALG, Backend, Config, EngineBackend, FitResult, Individual, SearchEngine,
                     SymbolicRegressor, variable_registry)

__all__ = ["BASIC", "LINALG", "Backend", "Config", "EngineBackend", "FitResult", "Individual", "SearchEngine",
           "SymbolicRegressor", "variable_registry"]
