/* orkan.h - umbrella header (reference include/orkan.h:4-9) plus the device extensions. */
#ifndef ORKAN_H
#define ORKAN_H

#include "q_types.h"
#include "state.h"
#include "gate.h"
#include "channel.h"
#include "meas.h"
#include "circ.h"
#include "orkan_dev.h"

#endif /* ORKAN_H */
