/* physics_oracle.c -- FP64 physics-mode oracle (filled in with the physics path). */
int orc_physics_version(void) { return 0; }
