# Minimal patch of hydro-cal-fortan/calculate.cpp (the reference CPU solver)
# so that decks with open boundaries run without undefined behaviour; applied
# by oracle/ref.mk to a copy under oracle/_ref/, never to the reference tree.
# Nothing else in the solver changes: its per-cell work is the same.
#
# 1. Each NQ series file is read into QZSTIME2 / QZSTEMP2, but the loop sizes
#    QZSTIME1 / QZSTEMP1 instead (calculate.cpp:1089-1096): size the buffers
#    that are filled.
/BOUNDE\/NQ\/NQ/,/QZSTEMP2\[i\];/{
s/QZSTIME1\.resize(NQTEMP, 0)/QZSTIME2.resize(NQTEMP, 0)/
s/QZSTEMP1\.resize(NQTEMP, 0)/QZSTEMP2.resize(NQTEMP, 0)/
}
# 2. ZT and QT are [boundary cell][day] (calculate.cpp:1052, :1079) but are
#    read as [day][cell] (:276, :320, :1170, :1176); read them in their own
#    order, with the last day's increment zero as the GPU reader has it
#    (mesh.cpp DZT/DQT loops).
s/QT\[jt\]\[II\]/QT[II][jt]/
s/ZT\[jt\]\[II\]/ZT[II][jt]/
s/DZT\[l\] = (ZT\[jt + 1\]\[l\] - ZT\[jt\]\[l\]) \/ K0;/DZT[l] = jt + 1 < NDAYS ? (ZT[l][jt + 1] - ZT[l][jt]) \/ K0 : 0.0;/
s/DQT\[l\] = (QT\[jt + 1\]\[l\] - QT\[jt\]\[l\]) \/ K0;/DQT[l] = jt + 1 < NDAYS ? (QT[l][jt + 1] - QT[l][jt]) \/ K0 : 0.0;/
# 3. BOUNDRYinterp reads one element past each series (:1110); stop at the
#    last interval.
s/for (int i = 0; i < NZQSTEMP; i++) {/for (int i = 0; i + 1 < NZQSTEMP; i++) {/
# 4. The boundary-group lists hold 1-based cell numbers, but CHOICE looks up
#    the 0-based cell (:275, :300, :319), so every lookup misses and indexes
#    one past the tables: look up the 1-based number.
s/CHOICE(\(MBQ\|MBZ\|MBZQ\), pos, II)/CHOICE(\1, pos + 1, II)/
# 5. A slot without neighbour has NAC = 0, so NC = NAC - 1 = -1, but the test
#    is NC == 0 (:124), which reads the state at index -1: test NC == -1, as
#    the GPU kernels do (functors.cu:98-106).
s/    if (NC == 0) {/    if (NC == -1) {/
