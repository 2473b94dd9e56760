/* <io.h> is not needed on Linux. */
