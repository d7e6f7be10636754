/* empty: stands in for the build configuration that the reference
 * generates with u.conf (src/inc/conf.h reads it); the hot-path device code
 * needs none of its switches */
