/* Forced include for the reference build (oracle/Makefile): glibc declares a global
 * `daylight` (time.h) that collides with the reference's `Spectrum daylight()`
 * (lights.h:32); rename the reference's symbol for this translation unit. */
#include <ctime>
#define daylight ft_daylight
