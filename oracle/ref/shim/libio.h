/* Empty stand-in: glibc no longer ships <libio.h>, which the reference's
 * src/IO/StreamGZ.hpp:32 includes without using anything from it. */
