"""CPU oracle of the baking substep: test infrastructure, never part of the product path."""
