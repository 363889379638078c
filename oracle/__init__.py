"""CPU oracle of the IBPM time step (test infrastructure only; never imported by the product)."""
