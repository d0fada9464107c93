/* The reference's tests/init.c calls two VAPOR converters (vdfcreate,
 * raw2vdf) from data2vdf/, which need VAPOR 2.3 libraries that are not
 * installed.  Only test_init() from that file is used here, so the two
 * converters are stubbed to report failure.  Test infrastructure only. */
int vdfcreate(int argc, char* argv[]) { (void)argc; (void)argv; return -1; }
int raw2vdf(int argc, char* argv[]) { (void)argc; (void)argv; return -1; }

/* init.c's VAPOR writer also prints the OpenMP thread count; the image's gcc
 * wrapper cannot link libgomp, so the writer's single query is stubbed. */
int omp_get_num_threads(void) { return 1; }
