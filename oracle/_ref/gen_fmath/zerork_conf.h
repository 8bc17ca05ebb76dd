#ifndef ZERORK_CONF_H
#define ZERORK_CONF_H
#endif
