/* placeholder until the 2D Helmholtz oracle lands */
