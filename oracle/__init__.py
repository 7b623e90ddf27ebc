"""CPU oracle of pyOCEAN's tracer hot path: test infrastructure, never part of the product path."""
