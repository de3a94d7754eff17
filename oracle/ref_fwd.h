/* Forced-include shim for compiling the unmodified reference with GCC 13:
 * include/bounce/dynamics/island.h names b3Contact and b3Joint before any
 * declaration is visible. Test infrastructure only (oracle build). */
#ifdef __cplusplus
class b3Contact;
class b3Joint;
#endif
