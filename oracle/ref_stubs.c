/* Link stub for building the reference's own src/main.c on the CPU path --
 * TEST INFRASTRUCTURE ONLY.  src/main.c:334 calls dt_destruct()
 * unconditionally; it is defined in the reference's CUDA engine
 * (new_dt_cuda.cu), which the CPU build does not compile, and has nothing
 * to release there. */
void dt_destruct(void) {}
