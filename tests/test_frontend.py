"""voxel_sql's parser on the CPU: the statement shapes the reference's
compiler handles (bindings/voxel_sql.py:48-316) parse into the structures the
executor reads; unsupported statements raise as the reference does."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "voxel_b200", "frontend"))

import voxel_sql as vsql  # noqa: E402


def parse(sql):
    return vsql._Parser(sql).statement()


def test_select_shapes():
    s = parse("SELECT SUM(price) FROM trades WHERE price > 500")
    assert s["targets"] == [("func", "sum", ("col", "price"))]
    assert s["from"] == ("table", "trades")
    assert s["where"] == ("cmp", ">", ("col", "price"), ("const", 500.0))
    s = parse("select count(*) as n from t where a >= -2.5e1 and (a < 3 or a = 7) group by k order by a desc limit 10;")
    assert s["targets"] == [("func", "count", ("star",))]
    assert s["where"][0] == "bool" and s["where"][1] == "and"
    assert s["where"][2][0] == ("cmp", ">=", ("col", "a"), ("const", -25.0))
    assert s["where"][2][1][1] == "or"
    assert s["group"] == ["k"] and s["sort"] is False and s["limit"] == ("const", 10.0)
    s = parse("SELECT * FROM 'data.csv' WHERE col > 100")
    assert s["from"] == ("table", "data.csv") and s["targets"] == [("star",)]
    s = parse("SELECT MAX(v) FROM (SELECT v FROM t LIMIT 3) AS sub")
    assert s["from"][0] == "subquery" and s["from"][1]["limit"] == ("const", 3.0)


def test_unsupported_statements():
    with pytest.raises(NotImplementedError):
        parse("INSERT INTO t VALUES (1)")
    with pytest.raises(NotImplementedError):
        parse("DELETE FROM t")
    with pytest.raises(ValueError):
        parse("")
    with pytest.raises(ValueError):
        vsql.execute("SELECT SUM(v) FROM missing_table", {})
    with pytest.raises(ValueError):
        vsql.execute("SELECT 1", {})
