/* crt_rand.c -- the rand() / srand() of the Microsoft C runtime, for the METIS build.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref/libstg_metis.so).  GKlib's random numbers come from
 * the C library's rand() unless USE_GKRAND is defined (GKlib/src/random.c:73-133), and the
 * reference's CMake never defines it (it sets GKRAND, which nothing reads).  The partitions
 * shipped in Assets/sorted_mesh were made by a Windows build, so METIS drew from the
 * Microsoft runtime's generator there; compiled against glibc's rand() the same METIS code
 * gives other partitions.  The METIS objects are compiled with rand / srand renamed to these
 * functions.  The generator is the runtime's documented linear congruential one:
 * state = state * 214013 + 2531011 (mod 2^32), value = bits 16..30 of the state (RAND_MAX
 * 0x7fff), seed 1 until srand is called. */
static unsigned int orc_crt_state = 1u;

void orc_crt_srand(unsigned int seed) { orc_crt_state = seed; }

int orc_crt_rand(void)
{
    orc_crt_state = orc_crt_state * 214013u + 2531011u;
    return (int)((orc_crt_state >> 16) & 0x7fffu);
}
