#ifndef ZERORK_CONF_H
#define ZERORK_CONF_H
#define ZERORK_EXP_LIBC 1
#endif
