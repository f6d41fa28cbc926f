/* TEST INFRASTRUCTURE ONLY: version header the reference build generates from
 * src/ConfigAPR.h.in (version 2.1.0 per CMakeLists.txt:46-48). */
#ifndef CONFIG_APR_H
#define CONFIG_APR_H
namespace ConfigAPR {
    const unsigned int APR_VERSION_MAJOR = 2;
    const unsigned int APR_VERSION_MINOR = 1;
    const unsigned int APR_VERSION_PATCH = 0;
    const char * const APR_GIT_HASH = "oracle";
    const char * const APR_VERSION = "2.1.0";
}
#endif
