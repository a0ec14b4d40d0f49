"""Design layer of the inverse-design loop: density -> permittivity maps
(filter, projection, erosion/dilation) on the GPU, the 3-D metalens problem,
and the plain and surrogate-assisted optimisation loops."""
