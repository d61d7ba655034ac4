#ifndef ACO_API_H
#define ACO_API_H
/* Symbols exported by libaco_b200.so (everything else is hidden). */
#if defined(__GNUC__)
#define ACO_API __attribute__((visibility("default")))
#else
#define ACO_API
#endif
#endif
