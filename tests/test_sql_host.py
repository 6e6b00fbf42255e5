"""The SQL front end on the CPU: the benchmark queries written as SQL over
the engine's tables map to their pipeline templates with the constants
they state, and what no template computes is refused with the reason."""
import pytest

from gpudbmetalcodegen_b200.engine import sql_to_spec
from gpudbmetalcodegen_b200._lib import GpudbError

Q1 = """
SELECT f_flag_a, f_flag_b, SUM(f_quantity) AS sum_qty, SUM(f_price) AS sum_base_price,
       SUM(f_price * (100 - f_discount)) AS sum_disc_price,
       SUM(f_price * (100 - f_discount) * (100 + f_tax)) AS sum_charge,
       AVG(f_quantity), AVG(f_price), AVG(f_discount), COUNT(*) AS count_order
FROM fact
WHERE f_ship_day <= 2436
GROUP BY f_flag_a, f_flag_b
ORDER BY f_flag_a, f_flag_b;
"""
Q6 = """select sum(f_price * f_discount) as revenue from fact
        where f_ship_day >= 365 and f_ship_day < 730 and f_discount between 5 and 7 and f_quantity < 24"""
Q3 = """SELECT p_fk, SUM(p_price * (100 - p_discount)) AS revenue
        FROM dim, probe
        WHERE b_key = p_fk AND b_segment = 1 AND b_order_day < 1170 AND p_ship_day > 1170
        GROUP BY p_fk ORDER BY revenue DESC, p_fk LIMIT 10"""


@pytest.mark.parametrize("sql,spec", [
    (Q1, "template=q1;ship_le=2436"),
    (Q1.replace("<= 2436", "< 2437"), "template=q1;ship_le=2436"),
    (Q6, "template=q6;ship_ge=365;ship_lt=730;disc_lo=5;disc_hi=7;qty_lt=24"),
    (Q6.replace("f_ship_day >= 365", "365 <= f_ship_day"), "template=q6;ship_ge=365;ship_lt=730;disc_lo=5;disc_hi=7;qty_lt=24"),
    (Q3, "template=join_topk;seg=1;od_lt=1170;ship_gt=1170;k=10"),
    (Q3.replace("ORDER BY revenue DESC", "ORDER BY SUM(p_price * (100 - p_discount)) DESC").replace("LIMIT 10", "LIMIT 32"),
     "template=join_topk;seg=1;od_lt=1170;ship_gt=1170;k=32"),
    (Q3.replace("p_ship_day > 1170", "p_ship_day >= 1171"), "template=join_topk;seg=1;od_lt=1170;ship_gt=1170;k=10"),
    ("select p_fk, p_price * (100 - p_discount) from probe, dim where p_fk = b_key and b_segment = 3 "
     "and b_order_day < 600 and p_ship_day > 500", "template=join_rows;seg=3;od_lt=600;ship_gt=500"),
    ("select z_key, count(*), sum(z_value) from zprobe group by z_key", "template=groupby"),
    ("select z_key, count(*), sum(zb_payload) from zbuild, zprobe where zb_key = z_key group by z_key order by z_key",
     "template=hashjoin"),
    ("select count(*), sum(m_value) from mix where m_filter < 5000", "template=mix_agg;thr=5000"),
    ("select m_rank_z % 1000, count(*), sum(m_value) from mix where m_filter < 5000 group by m_rank_z % 1000",
     "template=mix_groupby;key=m_rank_z;card=1000;thr=5000;groups=1000"),
    ("select m_rank_u % 64, sum(m_value) from mix where m_filter < 900 group by m_rank_u % 64 "
     "order by sum(m_value) desc, m_rank_u % 64 limit 5", "template=mix_topk;key=m_rank_u;card=64;thr=900;groups=64;k=5"),
    ("select count(*), sum(m_value) from mix, mixdim where m_fk = md_key and md_attr < 300 and m_filter < 7000",
     "template=mix_join;thr=7000;attr_lt=300"),
])
def test_benchmark_queries_map_to_their_templates(sql, spec):
    assert sql_to_spec(sql) == spec


@pytest.mark.parametrize("sql,why", [
    (Q6.replace(" and f_quantity < 24", ""), "f_quantity < <constant>"),
    (Q6.replace("f_quantity < 24", "f_quantity < 24 or f_tax = 1"), "OR is not supported"),
    (Q6.replace("5 and 7", "0.05 and 0.07"), "decimal literal"),
    (Q1.replace("COUNT(*)", "MAX(f_tax)"), "does not compute max(f_tax)"),
    (Q1.replace("ORDER BY f_flag_a, f_flag_b", "ORDER BY sum_qty DESC"), "ordered by its key columns"),
    (Q3.replace(" LIMIT 10", ""), "LIMIT 1..32"),
    (Q3.replace("DESC, p_fk", "ASC, p_fk"), "revenue descending"),
    (Q3.replace("b_key = p_fk AND ", ""), "join on b_key = p_fk"),
    (Q3.replace("b_segment = 1", "b_segment = 1 AND p_price > 7"), "no predicate like p_price"),
    ("select * from lineitem", "expected a name"),
    ("select x from nowhere", "no plan template reads"),
    ("select z_key from zprobe where", "expected a name"),
    ("select m_value % 10, count(*) from mix where m_filter < 5 group by m_value % 10", "grouped by m_rank_u %"),
    ("select count(*), sum(m_value) from mix", "m_filter < <constant>"),
    ("select m_rank_u % 8, sum(m_value) from mix where m_filter < 9 group by m_rank_u % 8 order by sum(m_value) limit 3",
     "sum(m_value) descending"),
])
def test_unmapped_queries_are_refused_with_the_reason(sql, why):
    with pytest.raises(GpudbError) as e:
        sql_to_spec(sql)
    assert why in e.value.message, e.value.message
