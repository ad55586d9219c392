/* Code-rate enum of the reference (reference include/enums.h:4-12), same
 * names and values so that reference call sites compile unchanged. */
#ifndef ENUMS_H
#define ENUMS_H

enum coderate
{
    HALFRATE = 0,
    TWOTHIRDSA = 1,
    TWOTHIRDSB = 2,
    THREEQUARTERSA = 3,
    THREEQUARTERSB = 4,
    FIVESIXTHS = 5
};

#endif
