/* The reference's tests/init.c calls two VAPOR converters (vdfcreate,
 * raw2vdf) from data2vdf/, which need VAPOR 2.3 libraries that are not
 * installed.  They are stubbed to do nothing and report success, so the
 * reference's own ring2d/ring3d drivers run (ring3d then leaves only its raw
 * per-field scratch file behind).  Test infrastructure only. */
int vdfcreate(int argc, char* argv[]) { (void)argc; (void)argv; return 0; }
int raw2vdf(int argc, char* argv[]) { (void)argc; (void)argv; return 0; }

/* init.c's VAPOR writer also prints the OpenMP thread count; the image's gcc
 * wrapper cannot link libgomp, so the writer's single query is stubbed. */
int omp_get_num_threads(void) { return 1; }
